// Test infrastructure: the REFERENCE's own GPU instance-tree build (src/cuda_tlas.cuh, neraulgraphics 0.5.0),
// compiled from its header where it lies with the reference's CUDA flags (-use_fast_math, CMakeLists.txt:127-131)
// by oracle/Makefile into oracle/_ref/libngref_tlas.so, and driven through one C entry point so the GPU tests can
// count how its keys, sorted order and tree differ from the product's. Nothing in the product links this file.
//
// ngref_tlas_build runs, on the default stream, exactly what tlas::Builder::build (cuda_tlas.cuh:255-276) runs,
// through the Builder itself, and then the header's own place_instances / make_keys kernels once more on
// buffers of its own for the keys in instance order (the Builder keeps its keys private; the kernels are the
// same launches on the same inputs, so the keys are the ones the Builder sorted).

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <neraulgraphics/renderer.h>

namespace {

[[noreturn]] void throw_cuda_error(const cudaError_t err, const char *call, const char *file, const int line) {
    throw std::runtime_error(std::string(file) + ":" + std::to_string(line) + ": " + call + " failed: " +
        cudaGetErrorString(err));
}

}  // namespace

#define CUDA_CHECK(call)                                                                \
    do {                                                                                \
        const cudaError_t err_ = (call);                                                \
        if (err_ != cudaSuccess) throw_cuda_error(err_, #call, __FILE__, __LINE__);     \
    } while (0)

#include "cuda_tlas.cuh"

namespace {

thread_local std::string g_error;

template <typename T>
struct Dev {
    T *p = nullptr;
    explicit Dev(size_t count) { CUDA_CHECK(cudaMalloc(&p, count * sizeof(T) + 16)); }
    ~Dev() { cudaFree(p); }
    Dev(const Dev &) = delete;
    Dev &operator=(const Dev &) = delete;
};

}  // namespace

extern "C" {

const char *ngref_tlas_last_error(void) { return g_error.c_str(); }

// worlds x per_world instances; local_bounds: per_world x 6 floats (each slot's mesh box in mesh space);
// matrices: n x 12 floats, world-major (host). Out (host, any may be NULL): keys (n, instance order), sorted_ids
// (n), nodes ((2n - 1) x 8 words, neraulgraphics::bvh::TlasNode), roots (worlds). Returns 0, or 2 with ngref_tlas_last_error().
int ngref_tlas_build(int worlds, int per_world, const float *local_bounds, const float *matrices, uint64_t *keys,
    int32_t *sorted_ids, int32_t *nodes, int32_t *roots) {
    using namespace neraulgraphics::device;
    try {
        const int n = worlds * per_world;
        const std::vector<float> lb(local_bounds, local_bounds + 6 * static_cast<size_t>(per_world));
        Dev<float> d_mat(12 * static_cast<size_t>(n));
        Dev<Instance> d_inst(n);
        CUDA_CHECK(cudaMemcpy(d_mat.p, matrices, 12 * static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice));
        tlas::Builder builder(worlds, per_world, lb);
        builder.build(d_mat.p, d_inst.p);
        CUDA_CHECK(cudaDeviceSynchronize());
        if (nodes)
            CUDA_CHECK(cudaMemcpy(nodes, builder.nodes, (2 * static_cast<size_t>(n) - 1) * sizeof(neraulgraphics::bvh::TlasNode),
                cudaMemcpyDeviceToHost));
        if (roots) CUDA_CHECK(cudaMemcpy(roots, builder.roots, static_cast<size_t>(worlds) * sizeof(int), cudaMemcpyDeviceToHost));
        if (sorted_ids) {
            std::vector<neraulgraphics::bvh::TlasNode> leaves(n);
            CUDA_CHECK(cudaMemcpy(leaves.data(), builder.nodes + (n - 1), static_cast<size_t>(n) * sizeof(neraulgraphics::bvh::TlasNode),
                cudaMemcpyDeviceToHost));
            for (int k = 0; k < n; ++k) sorted_ids[k] = ~leaves[k].left;
        }
        if (keys) {
            Dev<float> d_lb(lb.size()), d_aabb(6 * static_cast<size_t>(n));
            Dev<int> d_wb(6 * static_cast<size_t>(worlds)), d_ids(n);
            Dev<uint64_t> d_keys(n);
            CUDA_CHECK(cudaMemcpy(d_lb.p, lb.data(), lb.size() * sizeof(float), cudaMemcpyHostToDevice));
            constexpr int T = 128;
            tlas::init_world_bounds<<<(worlds + T - 1) / T, T>>>(d_wb.p, worlds);
            tlas::place_instances<<<(n + T - 1) / T, T>>>(d_mat.p, d_lb.p, per_world, n, d_inst.p, d_aabb.p, d_wb.p);
            tlas::make_keys<<<(n + T - 1) / T, T>>>(d_aabb.p, d_wb.p, per_world, n, d_keys.p, d_ids.p);
            CUDA_CHECK(cudaGetLastError());
            CUDA_CHECK(cudaMemcpy(keys, d_keys.p, static_cast<size_t>(n) * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        }
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 2;
    }
}

}  // extern "C"
