// sort_noalloc.cu -- the particle-key sort for callers that must not allocate.
//
// emerge_cuda_sort_keys allocates its device buffers and a stream per call.  Some
// callers cannot let a library do that: cudaMalloc/cudaFree synchronise the whole
// device (stalling the caller's other streams), and a caller whose memory pool has
// reserved the device's memory would see the allocation fail.  This entry point
// takes caller-owned device buffers and the caller's stream, and runs the same key
// kernel and stable radix sort over a fixed working array that lives in this
// library's device image, so it allocates nothing.  The array bounds the input
// size to EMERGE_SORT_NOALLOC_MAX positions.
#include <cuda.h>  // CUcontext / CUresult types only; the driver is reached through the runtime

#include <mutex>
#include <string>

#include "../../include/emerge_cuda.h"
#include "kernels.h"

namespace emerge {
void set_global_error(const char *msg);  // sim.cu: message for emerge_cuda_last_global_error
}

using namespace emerge;

namespace {

// Working space of one sort of up to EMERGE_SORT_NOALLOC_MAX (key, index) pairs:
// two key and two index ping-pong arrays (1 MiB at 65,536 pairs), the per-CTA digit
// histogram and the scan partials, 256-byte aligned pieces.  Nothing in it needs to
// start at zero: every pass writes each histogram entry and scan partial before
// reading it, and the key kernel writes the first key/index pair.
constexpr size_t kScratchBytes = size_t(1088) << 10;
static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;

// Address of the array on one device, with the id of the context it was looked up in: a
// context destroyed and created again (cudaDeviceReset) reloads the module, so the cached
// address is only reused while the device's current context is the same one.
struct ScratchEntry {
    void *ptr;
    unsigned long long ctx_id;
};
ScratchEntry g_scratch[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// Id of the calling thread's current context (cuCtxGetId: unique over the process's life,
// so a re-created context never repeats an old id).  False when there is no current context
// yet or the driver does not provide the entry points; callers then look the address up.
bool current_context_id(unsigned long long *id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {  // under g_setup_mutex
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        resolved = true;
    }
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

__global__ void k_copy_u32(const uint32_t *src, uint32_t *dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

emerge_status fail(emerge_status st, const std::string &msg) {
    set_global_error(msg.c_str());
    return st;
}

// True when `p` is device (or managed) memory usable from device `dev`.
bool device_accessible(const void *p, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // clear the query's error; it is reported as INVALID_ARG
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// Address of the scratch array on the current device, looked up once per device context.
emerge_status scratch_for_device(int dev, void **out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchEntry &entry = g_scratch[dev];
    unsigned long long id = 0;
    if (!(entry.ptr && current_context_id(&id) && id == entry.ctx_id)) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess)
            return fail(EMERGE_ERR_CUDA,
                        std::string("cudaGetSymbolAddress(sort scratch): ") + cudaGetErrorString(e));
        // the lookup made the device's context current; 0 (never a valid id) forces a new
        // lookup on the next call when the id cannot be read
        entry.ptr = p;
        entry.ctx_id = current_context_id(&id) ? id : 0ull;
    }
    *out = entry.ptr;
    return EMERGE_OK;
}

}  // namespace

extern "C" emerge_status emerge_cuda_sort_keys_noalloc(const float *xy_dev, uint32_t n,
                                                       uint32_t grid_res, int key_mode,
                                                       uint32_t *keys_dev, uint32_t *perm_dev,
                                                       void *stream) {
    // Everything rejectable is rejected before the first CUDA call.
    if (n > EMERGE_SORT_NOALLOC_MAX)
        return fail(EMERGE_ERR_INVALID_ARG, "sort_keys_noalloc: n = " + std::to_string(n) +
                                                " exceeds EMERGE_SORT_NOALLOC_MAX (" +
                                                std::to_string(EMERGE_SORT_NOALLOC_MAX) + ")");
    if ((key_mode != 0 && key_mode != 1) || grid_res < 1 || grid_res > 32768)
        return fail(EMERGE_ERR_INVALID_ARG,
                    "sort_keys_noalloc: key_mode must be 0 or 1 and grid_res in 1..32768");
    if (n == 0) return EMERGE_OK;
    if (!xy_dev || !keys_dev || !perm_dev || (reinterpret_cast<uintptr_t>(xy_dev) & 7u) ||
        (reinterpret_cast<uintptr_t>(keys_dev) & 3u) || (reinterpret_cast<uintptr_t>(perm_dev) & 3u))
        return fail(EMERGE_ERR_INVALID_ARG,
                    "sort_keys_noalloc: null or misaligned buffer (xy needs 8-byte, keys/perm "
                    "4-byte alignment)");
    // an error left pending by the caller's earlier work: not this call's failure
    const cudaError_t pending = cudaPeekAtLastError();
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(EMERGE_ERR_CUDA, std::string("sort_keys_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(EMERGE_ERR_UNSUPPORTED, "sort_keys_noalloc: device ordinal above 63");
    if (!device_accessible(xy_dev, dev) || !device_accessible(keys_dev, dev) ||
        !device_accessible(perm_dev, dev))
        return fail(EMERGE_ERR_INVALID_ARG,
                    "sort_keys_noalloc: xy, keys and perm must be device memory of the current "
                    "device (or managed memory)");

    void *base = nullptr;
    emerge_status st = scratch_for_device(dev, &base);
    if (st != EMERGE_OK) return st;
    if (sort_scratch_bytes(EMERGE_SORT_NOALLOC_MAX) > kScratchBytes)
        return fail(EMERGE_ERR_CUDA, "sort_keys_noalloc: scratch array smaller than the sort needs");
    SortScratch sc;
    sort_scratch_bind(sc, base, EMERGE_SORT_NOALLOC_MAX);

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int ni = static_cast<int>(n);
    const int blocks = (ni + 255) / 256;
    launch_sort_keys(reinterpret_cast<const float2 *>(xy_dev), ni, static_cast<int>(grid_res),
                     key_mode, sc.keys[0], sc.vals[0], s);
    k_copy_u32<<<blocks, 256, 0, s>>>(sc.keys[0], keys_dev, ni);
    int r = radix_sort_pairs(sc, ni, sort_key_bits(static_cast<int>(grid_res), key_mode), s);
    k_copy_u32<<<blocks, 256, 0, s>>>(sc.vals[r], perm_dev, ni);
    e = cudaPeekAtLastError();
    if (e != cudaSuccess && e != pending)
        return fail(EMERGE_ERR_CUDA, std::string("sort_keys_noalloc: launch: ") + cudaGetErrorString(e));
    return EMERGE_OK;
}
