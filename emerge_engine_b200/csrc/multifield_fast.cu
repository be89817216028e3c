// multifield_fast.cu -- the fast pipeline's contact resolve (grid/contact.rs:254-391):
// grip cells holding one field take the total velocity, the interface cells are resolved
// one warp per cell from the particle pass's base-cell point lists.  Compiled like the fast
// translation unit (FMA contraction, approximate division and square root).
#define EMERGE_FAST_TU 1
#include "multifield.cuh"

namespace emerge {

namespace {

// First kernel: every grip cell that holds one field only resolves to the total velocity
// (contact.rs:303-307) and needs no point cloud; the cells holding both fields (the
// interface) are listed for the warp-per-cell kernel.
__global__ void k_contact_cells(GridView g, StepState *st) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    const float4 gr = g.acc_grip[ci];
    if (!(gr.w > 0.0f)) return;  // not in the grip field
    const float rest_mass = gr.w < 1.5f ? 0.0f : g.grid_m[ci] - gr.x;  // w = 1: grip only
    if (gr.x <= 1.0e-6f || rest_mass <= 1.0e-6f) {
        g.grip_v[ci] = g.grid_v[ci];
        g.rest_v[ci] = g.grid_v[ci];
        return;
    }
    g.iface[atomicAdd(&st->n_iface, 1u)] = static_cast<int>(k);
}

// Second kernel: one warp per interface cell.  The points on the lists the previous particle
// pass built (parity acc_slot ^ 1) are gathered into shared memory by nine lanes, one per
// base cell, and the fit's sums are split over the warp; a cell with more points than the
// buffer holds is resolved by lane 0 walking the lists.
constexpr int IFACE_WARPS = 8;
constexpr int IFACE_POINTS = 192;
__global__ void __launch_bounds__(IFACE_WARPS * 32) k_contact_iface(GridView g, DevConfig cfg, StepState *st,
                                                                   int n_particles) {
    __shared__ float4 s_pts[IFACE_WARPS][IFACE_POINTS];
    __shared__ int s_n[IFACE_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_cells = static_cast<int>(st->n_iface);
    const int *head = g.chead[st->acc_slot ^ 1u];
    for (int c = blockIdx.x * IFACE_WARPS + warp; c < n_cells; c += gridDim.x * IFACE_WARPS) {
        const int k = g.iface[c];
        const int x = k / g.res, y = k % g.res;
        const int ci = cell_index(x, y, g.tpd);
        const float4 gr = g.acc_grip[ci];
        if (lane == 0) s_n[warp] = 0;
        __syncwarp();
        if (lane < 9) {
            const int bx = x + lane / 3 - 1, by = y + lane % 3 - 1;
            if (in_domain(bx, by, g.res)) {
                int visited = 0;
                for (int j = head[bx * g.res + by]; j >= 0;) {
                    if (j >= n_particles || ++visited > n_particles) {
                        atomicOr(&st->error_flags, ERR_CONTACT_LIST);
                        break;
                    }
                    const float4 q = g.cpts[j];
                    const int slot = atomicAdd(&s_n[warp], 1);
                    if (slot < IFACE_POINTS) s_pts[warp][slot] = q;
                    j = __float_as_int(q.w);
                }
            }
        }
        __syncwarp();
        const int n = s_n[warp];
        if (n <= IFACE_POINTS) {
            contact_resolve_cell(g, cfg, st, x, y, ci, gr, WarpPoints{s_pts[warp], n, lane});
        } else if (lane == 0) {
            contact_resolve_cell(g, cfg, st, x, y, ci, gr,
                                 ListPoints(head, g.cpts, g.res, x, y, n_particles, &st->error_flags));
        }
        __syncwarp();
    }
}

}  // namespace

// The interface kernel's grid: four CTAs per SM of the current device (its warps stride over
// the interface cells, whose count is known only on the device).
static int iface_blocks() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        sms = 148;
    return 4 * sms;
}

void launch_contact_resolve_lists(const StepLaunch &L) {
    k_contact_cells<<<grid_blocks(L.g), MF_THREADS, 0, L.stream>>>(L.g, L.st);
    k_contact_iface<<<iface_blocks(), IFACE_WARPS * 32, 0, L.stream>>>(L.g, L.cfg, L.st, L.n);
}

}  // namespace emerge
