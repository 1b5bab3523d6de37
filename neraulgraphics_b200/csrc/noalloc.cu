// A tree build for callers that cannot allocate device memory.
//
// Who needs it: frameworks that reserve most of the GPU for their own memory pool up front (JAX's
// preallocation, for one) may find a stray cudaMalloc fails or fragments their pool. Such a caller owns
// every input and output buffer already, but the build also needs scratch space (each node's parent and an
// arrival counter per internal node), which the renderer otherwise allocates with cudaMalloc.
//
// Here that scratch is a file-scope static device array of fixed size, so calls allocate nothing. Limits and
// rules:
//   - at most NOALLOC_MAX_INSTANCES instances over all worlds (and at most 1024 per world); larger calls are
//     rejected with NGB_INVALID_ARGUMENT before anything is queued;
//   - every GPU that loads this library holds the array (about 0.8 MB) until the process exits;
//   - the array's device address is looked up by the first call made in a CUDA context (a device's primary
//     context, or one the caller made current), and again whenever the calling thread's current context is
//     a different one (after cudaDeviceReset, say);
//   - every call shares the one array: two calls whose work overlaps on the GPU (different streams, or
//     different host threads, without ordering between them) race and corrupt each other's trees. Order them
//     on one stream, or serialise them;
//   - a build whose bottom-up climb runs past the step limit a valid tree allows (malformed links) stops the
//     climb and writes a nonzero code to the caller's error word, when one is given.
#include <cuda.h>  // driver types only: the driver's calls are found at run time, nothing links libcuda

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/ngb.h"
#include "kernels.h"

namespace ngb {
void set_global_error(const std::string &message);  // renderer.cpp: what ngb_last_error(NULL) returns
}

namespace {

constexpr long long NOALLOC_MAX_INSTANCES = 65536;
constexpr long long PARENT_OFFSET = 0;                                  // 2n - 1 parent links
constexpr long long ARRIVALS_OFFSET = 2 * NOALLOC_MAX_INSTANCES;        // n - 1 arrival counters
constexpr long long ERROR_OFFSET = 3 * NOALLOC_MAX_INSTANCES;           // the kernels' error word
constexpr long long SCRATCH_INTS = 3 * NOALLOC_MAX_INSTANCES + 64;

static __device__ __align__(256) int g_tlas_scratch[SCRATCH_INTS];

// The array's address per CUDA context, keyed by the context's process-unique ID (cuCtxGetId), so a
// context that was destroyed and made again (cudaDeviceReset) is looked up afresh.
constexpr int MAX_CONTEXTS = 64;
struct Known {
    unsigned long long context_id;
    int *address;
};
std::mutex g_setup_mutex;
Known g_known[MAX_CONTEXTS] = {};
int g_known_count = 0;

using CtxGetCurrent = CUresult (*)(CUcontext *);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long *);

// The current context's unique ID, through the driver's entry points as the runtime hands them out.
cudaError_t current_context_id(unsigned long long *id) {
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2);
        if (e != cudaSuccess) return e;
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f || !g)
            return cudaErrorNotSupported;
        get_current = reinterpret_cast<CtxGetCurrent>(f);
        get_id = reinterpret_cast<CtxGetId>(g);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return cudaErrorDeviceUninitialized;
    return get_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorContextIsDestroyed;
}

int fail(int status, const std::string &message) {
    ngb::set_global_error(message);
    return status;
}

}  // namespace

extern "C" int ngb_build_tlas_noalloc(int32_t world_count, int32_t instances_per_world, const float *matrices,
    const float *slot_bounds, const int32_t *slot_blas_root, float *instance_records, uint64_t *keys,
    int32_t *sorted_ids, float *tlas_nodes, int32_t *roots, int32_t *error_word, void *stream) {
    const long long n = static_cast<long long>(world_count) * instances_per_world;
    if (world_count < 1 || instances_per_world < 1)
        return fail(NGB_INVALID_ARGUMENT, "world_count and instances_per_world must be 1 or more");
    if (instances_per_world > ngb::MAX_PER_WORLD)
        return fail(NGB_INVALID_ARGUMENT, "a world holds " + std::to_string(instances_per_world) + " instances, at most " +
            std::to_string(ngb::MAX_PER_WORLD) + " fit the per-world tree build");
    if (n > NOALLOC_MAX_INSTANCES)
        return fail(NGB_INVALID_ARGUMENT, std::to_string(n) + " instances over all worlds do not fit the static scratch "
            "of ngb_build_tlas_noalloc, which holds at most " + std::to_string(NOALLOC_MAX_INSTANCES));
    if (!matrices || !slot_bounds || !slot_blas_root || !instance_records || !keys || !sorted_ids || !tlas_nodes || !roots)
        return fail(NGB_INVALID_ARGUMENT, "no array given to ngb_build_tlas_noalloc may be null (but error_word)");
    if ((reinterpret_cast<uintptr_t>(instance_records) | reinterpret_cast<uintptr_t>(tlas_nodes)) & 15)
        return fail(NGB_INVALID_ARGUMENT, "instance_records and tlas_nodes must be 16-byte aligned");
    if (reinterpret_cast<uintptr_t>(keys) & 7) return fail(NGB_INVALID_ARGUMENT, "keys must be 8-byte aligned");
    if (reinterpret_cast<uintptr_t>(error_word) & 3) return fail(NGB_INVALID_ARGUMENT, "error_word must be 4-byte aligned");

    int *scratch = nullptr;
    {
        // Once per context, with it current: the host-side name of the array is not a device address, so the
        // address comes from the runtime.
        unsigned long long id = 0;
        cudaError_t e = current_context_id(&id);
        if (e == cudaErrorDeviceUninitialized) {
            // No context is current on this thread yet: the runtime's symbol lookup makes the current device's
            // primary context current.
            e = cudaGetSymbolAddress(reinterpret_cast<void **>(&scratch), g_tlas_scratch);
            if (e == cudaSuccess) e = current_context_id(&id);
        }
        if (e != cudaSuccess)
            return fail(NGB_CUDA_ERROR, std::string("finding the current CUDA context failed: ") + cudaGetErrorString(e));
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        int *known = nullptr;
        for (int k = 0; k < g_known_count; ++k)
            if (g_known[k].context_id == id) known = g_known[k].address;
        if (known) {
            scratch = known;
        } else {
            if (!scratch) e = cudaGetSymbolAddress(reinterpret_cast<void **>(&scratch), g_tlas_scratch);
            if (e != cudaSuccess)
                return fail(NGB_CUDA_ERROR, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            g_known[g_known_count < MAX_CONTEXTS ? g_known_count++ : static_cast<int>(id % MAX_CONTEXTS)] = Known{id, scratch};
        }
    }
    cudaError_t e = cudaSuccess;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The array keeps the last call's contents: the root's parent link, the arrival counters and the error
    // word (the caller's, or the array's own) must start this build at -1, 0 and 0.
    int *parent = scratch + PARENT_OFFSET, *arrivals = scratch + ARRIVALS_OFFSET;
    int *error = error_word ? error_word : scratch + ERROR_OFFSET;
    if ((e = cudaMemsetAsync(parent, 0xFF, sizeof(int), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(arrivals, 0, static_cast<size_t>(n > 1 ? n - 1 : 1) * sizeof(int), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(error, 0, sizeof(int), s)) != cudaSuccess)
        return fail(NGB_CUDA_ERROR, std::string("cudaMemsetAsync failed: ") + cudaGetErrorString(e));

    ngb::BuildArgs a{};
    a.worlds = world_count;
    a.per_world = instances_per_world;
    a.n = n;
    a.compose = 0;
    a.matrices_in = matrices;
    a.matrices_out = nullptr;
    a.slot_bounds = slot_bounds;
    a.slot_blas_root = slot_blas_root;
    a.inst = reinterpret_cast<float4 *>(instance_records);
    a.keys = reinterpret_cast<unsigned long long *>(keys);
    a.sorted_ids = sorted_ids;
    a.tlas = reinterpret_cast<float4 *>(tlas_nodes);
    a.roots = roots;
    a.parent = parent;
    a.arrivals = arrivals;
    a.error_flag = error;
    e = ngb::launch_build_worlds(a, s);
    if (e != cudaSuccess) return fail(NGB_CUDA_ERROR, std::string("launching the tree build failed: ") + cudaGetErrorString(e));
    ngb::set_global_error("");
    return NGB_OK;
}
