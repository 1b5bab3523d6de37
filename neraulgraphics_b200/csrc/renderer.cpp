// The renderer behind the C ABI (include/ngb.h): validation, device buffers, the stream, launches and
// bounded waits. Replaces BatchRenderer (src/batch.cpp) over CudaBackend (src/cuda_backend.cu:325-793).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "host.h"
#include "kernels.h"

namespace ngb {

[[noreturn]] void cuda_fail(cudaError_t e, const char *call, const char *file, int line) {
    throw CudaFailure(static_cast<int>(e), std::string(file) + ":" + std::to_string(line) + ": " + call + " failed: " +
        cudaGetErrorString(e) + " (" + cudaGetErrorName(e) + ")");
}
#define CK(call)                                                                 \
    do {                                                                         \
        const cudaError_t err_ = (call);                                         \
        if (err_ != cudaSuccess) ngb::cuda_fail(err_, #call, __FILE__, __LINE__); \
    } while (0)

// What the kernels' error flag means. It stays set: the renderer's later results are not trusted.
std::string device_error_message(int code) {
    switch (code) {
    case 1: return "a traversal stack overflowed; the images of that call are incomplete";
    case 2: return "a tree walk ran longer than the tree allows (malformed tree); the images are incomplete";
    case 3: return "a world's box refit ran longer than its tree allows (malformed tree)";
    case 4: return "the refit of the inter-world nodes ran longer than the tree allows (malformed tree)";
    default: return "the GPU kernels reported error " + std::to_string(code);
    }
}

namespace {

// A named range around a call's host work and launches on Nsight timelines (nothing without a tool attached).
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

// Bytes held by every renderer's device arrays, and the host-side allocation-failure injection for tests:
// the value-th device allocation from now on fails (0: the next one), -1 none.
std::atomic<long long> g_device_bytes{0};
std::atomic<long long> g_fail_allocation{-1};

bool injected_allocation_failure() {
    long long v = g_fail_allocation.load();
    while (v >= 0)
        if (g_fail_allocation.compare_exchange_weak(v, v - 1)) return v == 0;
    return false;
}

// A device array, grown on demand and freed with its owner.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            cudaFree(p);
            g_device_bytes -= static_cast<long long>(n * sizeof(T));
        }
        p = nullptr;
        n = 0;
    }
    // At least count elements; the old contents are not kept when it grows.
    T *ensure(size_t count) {
        if (count == 0) return p;
        if (p && count <= n) return p;
        release();
        if (injected_allocation_failure())
            cuda_fail(cudaErrorMemoryAllocation, "cudaMalloc (a failure injected by ngb_inject_allocation_failure)",
                __FILE__, __LINE__);
        CK(cudaMalloc(&p, count * sizeof(T)));
        n = count;
        g_device_bytes += static_cast<long long>(n * sizeof(T));
        return p;
    }
};

// Makes the renderer's GPU current for the call and restores the caller's afterwards.
struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        CK(cudaGetDevice(&previous));
        if (previous != device) CK(cudaSetDevice(device));
    }
    ~DeviceGuard() {
        int now = -1;
        if (cudaGetDevice(&now) == cudaSuccess && now != previous && previous >= 0) cudaSetDevice(previous);
    }
};

DevMaterial dev_material(const ngb_material &m) {
    return DevMaterial{make_float3(m.diffuse_color.x, m.diffuse_color.y, m.diffuse_color.z), m.diffuse_albedo,
        m.specular_albedo, m.reflectivity, m.specular_exponent, 0.0f};
}

}  // namespace

// Worlds of uneven instance counts and image sizes (one camera each), as ngb_create_uneven lays them out.
struct UnevenLayout {
    std::vector<int> first;          // world w's instances are [first[w], first[w + 1])
    std::vector<int> width, height;  // its image
};

struct Renderer {
    std::mutex mutex;
    std::string last_error;
    int width = 0, height = 0, worlds = 0, cpw = 0, per_world = 0, device = 0;
    long long n = 0;
    SceneParams params{};
    // The rows every render draws, [band_first, band_first + band_rows) of each view's image (ngb_set_rows):
    // the whole image by default.
    int band_first = 0, band_rows = 0;

    // The scene: shared meshes and what each slot of a world holds.
    DevBuf<float4> blas, tris, attrs;
    DevBuf<int> tri_index, slot_blas_root;
    DevBuf<int> tri_of_local, slot_tri_base;  // a mesh-local triangle's packed index, for the adjoint
    DevBuf<float> slot_bounds;
    DevBuf<DevMaterial> slot_material;
    // Per build.
    DevBuf<float> matrices;
    DevBuf<float4> inst, tlas;
    DevBuf<unsigned long long> keys;
    DevBuf<int> sorted_ids, roots, parent, arrivals, leaf_of;
    DevBuf<float4> slot_hull, slot_sphere;
    // The global build's scratch (worlds of more than MAX_PER_WORLD instances, or when asked for).
    int build_mode = 0;  // 0: automatic, 1: the per-world build, 2: the global build
    DevBuf<float4> large_aabb;
    DevBuf<int> large_bounds, large_ids_a, large_ids_b;
    DevBuf<unsigned long long> large_keys_a, large_keys_b;
    DevBuf<unsigned> large_counts;
    DevBuf<float4> blas_pairs, tlas_pairs;
    DevBuf<int2> slot_root;
    DevBuf<unsigned long long> work_counter;  // the persistent render's job counter
    DevBuf<float4> camera_basis;              // the persistent and tile renders' per-view cameras
    DevBuf<float4> pic_hit, shadow_o, shadow_d;  // the tile render's per-pixel hand-over between its kernels
    DevBuf<int> pic_code, shadow_self;
    DevBuf<int> view_order;                   // the tile render's per-view candidate order, and its bounds
    DevBuf<float> view_bound;
    DevBuf<float> srgb_table;                 // 256 sRGB byte thresholds
    // Single-view renders (ngb_render_view): the running sums of the picture (zeroed when made, so a first render
    // with frame > 0 adds to zero), this frame's radiance, and the average's 0xAARRGGBB pixels.
    DevBuf<float4> view_accum, view_radiance;
    DevBuf<uint32_t> view_argb;
    bool reflective = false;                  // some material bounces light (reflectivity >= 1e-3)
    int kernel_choice = 0;                    // 0: automatic, 1: per pixel, 2: persistent, 3: tiles
    int ray_kernel = 0;                       // ray queries: 0 automatic, 1 per thread, 2 persistent, 3 packets
    PersistentTuning tuning{128, 28, 72, 16};
    PersistentTuning tile_tuning{128, 0, 56, 0};
    // Ray queries: the persistent kernel's shape measured best for them (no leaf batching), unless the caller
    // chose the persistent kernel and its shape.
    PersistentTuning ray_tuning{256, 28, 64, 1};
    // Bodies.
    bool bound = false;
    int bodies_per_world = 0;
    DevBuf<int> body_of_instance;
    DevBuf<float> local_pose, local_scale, body_poses;
    // Geoms carrying the instances (bind_geoms): per slot its geom and scale, and host poses' device copies.
    int geoms_per_world = 0;
    bool geoms_bound = false;
    DevBuf<int> geom_of_instance;
    DevBuf<float> geom_scale, geom_xpos, geom_xmat;
    // Meshes whose vertices change (update_mesh): per mesh its first node (its node capacity is 2T - 1), first
    // packed triangle, triangle and vertex counts, current node count, and where its indices and kept vertex
    // normals are in mesh_indices / mesh_normals (-1: none); per slot its mesh. The device rebuild's scratch.
    std::vector<int> mesh_node_base, mesh_tri_base, mesh_tris, mesh_verts, mesh_nodes, mesh_index_at, mesh_normal_at;
    DevBuf<uint32_t> mesh_indices;
    DevBuf<float> mesh_normals, mesh_stage;
    DevBuf<int> slot_mesh;
    std::vector<int> slot_mesh_host;
    DevBuf<float> mb_box, mb_centre, mb_node_box;
    DevBuf<uint32_t> mb_order;
    DevBuf<int> mb_lpos, mb_rpos, mb_begin, mb_end, mb_left, mb_depth, mb_index, mb_counter, mb_starts, mb_top, mb_prefix;
    DevBuf<int> mb_level_count;
    int *host_count = nullptr;  // pinned: a level's node count read back during a mesh rebuild
    // Staging for host inputs and the renderer's own outputs.
    DevBuf<float> cameras, ray_origins, ray_directions;
    DevBuf<uint8_t> out_rgb;
    DevBuf<float> out_depth, out_normal;
    DevBuf<int32_t> out_id;
    DevBuf<float> ray_distance, ray_normal;
    DevBuf<int32_t> ray_id;
    bool record_hits = false;
    DevBuf<int32_t> hit_instance, hit_triangle;
    DevBuf<float> hit_u, hit_v;
    // The caller's hit arrays (ngb_record_hits_into), written instead of the renderer's own while set.
    int32_t *ext_instance = nullptr, *ext_triangle = nullptr;
    float *ext_u = nullptr, *ext_v = nullptr;
    // The arrays the last render's hits went to (the caller's or the renderer's own).
    const int32_t *hits_instance() const { return ext_instance ? ext_instance : hit_instance.p; }
    const int32_t *hits_triangle() const { return ext_instance ? ext_triangle : hit_triangle.p; }
    const float *hits_u() const { return ext_instance ? ext_u : hit_u.p; }
    const float *hits_v() const { return ext_instance ? ext_v : hit_v.p; }
    DevBuf<int> error_flag;
    int *host_error = nullptr;  // pinned: the device error flag, copied back where the host waits for the work

    bool cuda_touched = false;  // set before the first CUDA call of the constructor
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_done = nullptr;
    cudaEvent_t ev_stage[2] = {nullptr, nullptr};  // between the tile render's camera, shade and shadow kernels
    int stages = 0;                                // kernels timed apart in the last render: 1 or 3
    float stage_ms[3] = {0.0f, 0.0f, 0.0f};
    bool synchronous = true;
    double timeout = 120.0;
    float kernel_ms = 0.0f;
    bool timing_pending = false;

    // Uneven worlds: per-world instance ranges, per-view image sizes and offsets (see ngb_create_uneven).
    bool uneven = false;
    std::vector<int> world_first_host;
    DevBuf<int> world_first;
    DevBuf<int4> view_info;
    DevBuf<int> view_pair_tile;  // per view: its first 4 x 4 tile (the camera kernel's paired tiles)
    long long total_pair_tiles = 0;
    long long total_pixels = 0, total_tiles = 0;

    explicit Renderer(const ngb_scene &s, const UnevenLayout *layout = nullptr);
    ~Renderer();
    void init(const ngb_scene &s, const UnevenLayout *layout);
    void teardown();

    void build(const float *matrices_in, int compose, const float *poses, const float *xmat = nullptr);
    void queue_error_read();
    void finish();
    void read_timing();
    // Whether the stream is being captured into a CUDA graph.
    bool capturing() const {
        cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
        return cudaStreamIsCapturing(stream, &status) == cudaSuccess && status != cudaStreamCaptureStatusNone;
    }
    bool use_large_build() const { return build_mode == 2 || (build_mode == 0 && per_world > MAX_PER_WORLD); }
    void wait(cudaEvent_t ev, double seconds);
    void set_instance_transforms(const float *m, int memory);
    void bind_bodies(int bpw, const int32_t *boi, const float *lp, const float *sc);
    void set_body_poses(const float *poses, int memory);
    void bind_geoms(int gpw, const int32_t *goi, const float *sc);
    void update_mesh(int mesh, const float *vertices, const float *normals, int memory);
    void set_geom_poses(const float *xpos, const float *xmat, int memory);
    void check_render(const float *cams, float fov, int spp, unsigned outputs, int frame, int memory);
    void render(const float *cams, float fov, int spp, unsigned outputs, int frame, int memory, uint8_t *rgb,
        float *depth, float *normal, int32_t *ids, const ngb_camera *view = nullptr);
    void check_view(const ngb_camera *camera, int frame, int spp);
    void put_lights(const ngb_light *lights, int count);
    void cast_rays(const float *o, const float *d, int rays_per_world, float max_distance, int memory, ngb_ray_hits *out,
        float *distance, float *normal, int32_t *ids);
    int rows() const { return band_rows > 0 ? band_rows : height; }
    size_t pixels() const {
        return uneven ? static_cast<size_t>(total_pixels) : static_cast<size_t>(worlds) * cpw * rows() * width;
    }
    int world_of_instance(long long g) const {
        if (!uneven) return static_cast<int>(g / per_world);
        return static_cast<int>(std::upper_bound(world_first_host.begin(), world_first_host.end(), g) -
            world_first_host.begin()) - 1;
    }
};

// A constructor that fails part way frees what it made (src/cuda_backend.cu:210-323 does the same).
Renderer::Renderer(const ngb_scene &s, const UnevenLayout *layout) {
    try {
        init(s, layout);
    } catch (...) {
        teardown();
        throw;
    }
}

Renderer::~Renderer() { teardown(); }

void Renderer::init(const ngb_scene &s, const UnevenLayout *layout) {
    if (layout) {
        // The shared scene is checked as it is; each world's image and instance range on their own.
        uneven = true;
        const int W = static_cast<int>(layout->width.size());
        require(W >= 1, "world_count must be 1 or more, got " + std::to_string(W));
        require(layout->first.back() == s.instance_count, "the worlds' instance counts add up to " +
            std::to_string(layout->first.back()) + ", but the scene lists " + std::to_string(s.instance_count));
        for (int w = 0; w < W; ++w) {
            check_frame_size(layout->width[w], layout->height[w]);
            const int count = layout->first[w + 1] - layout->first[w];
            require(count >= 0 && count <= TILE_MAX_INSTANCES, "world " + std::to_string(w) + " holds " +
                std::to_string(count) + " instances; uneven worlds hold 0 to " + std::to_string(TILE_MAX_INSTANCES));
            total_pixels += static_cast<long long>(layout->width[w]) * layout->height[w];
        }
        require(total_pixels <= INT32_MAX, "the worlds' images hold " + std::to_string(total_pixels) +
            " pixels, at most 2^31 - 1 are supported");
    } else {
        check_frame_size(s.width, s.height);
        require(s.world_count >= 1, "world_count must be 1 or more, got " + std::to_string(s.world_count));
        require(s.cameras_per_world >= 1, "cameras_per_world must be 1 or more, got " + std::to_string(s.cameras_per_world));
        const long long views = static_cast<long long>(s.world_count) * s.cameras_per_world;
        require(views * s.height <= INT32_MAX, std::to_string(views) + " views of height " + std::to_string(s.height) +
            " are too many");
    }
    check_scene(s);
    check_meshes(s);
    if (!layout) {
        require(s.instance_count <= MAX_INSTANCES_PER_WORLD, "a world holds " + std::to_string(s.instance_count) +
            " instances, at most " + std::to_string(MAX_INSTANCES_PER_WORLD) + " are supported");
        require(static_cast<long long>(s.world_count) * s.instance_count <= (INT32_MAX - 1) / 2,
            "too many instances over all worlds");
    }
    int device_count = 0;
    CK(cudaGetDeviceCount(&device_count));
    require(s.device >= 0 && s.device < device_count, "device " + std::to_string(s.device) + " does not exist");
    device = s.device;
    if (layout) {
        width = height = 0;
        worlds = static_cast<int>(layout->width.size());
        cpw = 1;
        world_first_host = layout->first;
        per_world = 0;
        for (int w = 0; w < worlds; ++w) per_world = std::max(per_world, layout->first[w + 1] - layout->first[w]);
        n = s.instance_count;
    } else {
        width = s.width;
        height = s.height;
        worlds = s.world_count;
        cpw = s.cameras_per_world;
        per_world = s.instance_count;
        n = static_cast<long long>(worlds) * per_world;
    }
    DeviceGuard guard(device);
    cuda_touched = true;
    CK(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;
    CK(cudaEventCreate(&ev_start));
    CK(cudaEventCreate(&ev_stop));
    CK(cudaEventCreate(&ev_stage[0]));
    CK(cudaEventCreate(&ev_stage[1]));
    CK(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    CK(cudaHostAlloc(&host_error, sizeof(int), cudaHostAllocDefault));
    CK(cudaHostAlloc(&host_count, sizeof(int), cudaHostAllocDefault));
    *host_error = 0;
    error_flag.ensure(1);
    CK(cudaMemsetAsync(error_flag.p, 0, sizeof(int), stream));

    // The classic scene: spheres, lights (as the reference's to_device: src/device_scene.h:265-272), floor, sky.
    for (int i = 0; i < s.sphere_count; ++i) {
        const ngb_sphere &sp = s.spheres[i];
        params.spheres[i] = DevSphere{make_float3(sp.center.x, sp.center.y, sp.center.z), sp.radius, dev_material(sp.material)};
    }
    put_lights(s.lights, s.light_count);
    params.sphere_count = s.sphere_count;
    // A path bounces when throughput * reflectivity >= 1e-3 (src/render_core.h:238-239); with throughput 1
    // at the first hit, that is any material hit with reflectivity >= 1e-3.
    for (int i = 0; i < s.sphere_count; ++i) reflective = reflective || s.spheres[i].material.reflectivity >= 1e-3f;
    reflective = reflective || (s.floor.half_extent_x > 0.0f && s.floor.material.reflectivity >= 1e-3f);
    for (int i = 0; i < s.instance_count; ++i) reflective = reflective || s.instances[i].material.reflectivity >= 1e-3f;
    work_counter.ensure(1);
    {
        float table[256];
        srgb_thresholds(table);
        srgb_table.ensure(256);
        CK(cudaMemcpy(srgb_table.p, table, sizeof(table), cudaMemcpyHostToDevice));
        params.srgb_table = srgb_table.p;
    }
    params.floor = DevPlane{s.floor.y, s.floor.half_extent_x, s.floor.z_min, s.floor.z_max, s.floor.checker_scale,
        dev_material(s.floor.material)};
    params.env_up = make_float3(0.0f, 1.0f, 0.0f);
    params.env_color_up = make_float3(0.10f, 0.26f, 0.60f);
    params.env_color_down = make_float3(0.35f, 0.52f, 0.70f);
    params.env_intensity = 1.0f;
    params.ambient = 0.0f;
    params.instance_count = static_cast<int>(n);
    params.per_world = per_world;
    if (uneven) {
        // Per view: (width, height, first pixel, first tile of 8 x 4 pixels).
        std::vector<int4> info(worlds);
        std::vector<int> pair_first(worlds);
        long long pix = 0, tile = 0, pair_tile = 0;
        for (int w = 0; w < worlds; ++w) {
            const int vw = layout->width[w], vh = layout->height[w];
            info[w] = make_int4(vw, vh, static_cast<int>(pix), static_cast<int>(tile));
            pair_first[w] = static_cast<int>(pair_tile);
            pix += static_cast<long long>(vw) * vh;
            tile += static_cast<long long>((vw + 7) / 8) * ((vh + 3) / 4);
            pair_tile += static_cast<long long>((vw + 3) / 4) * ((vh + 3) / 4);
        }
        total_tiles = tile;
        total_pair_tiles = pair_tile;
        view_info.ensure(worlds);
        CK(cudaMemcpy(view_info.p, info.data(), info.size() * sizeof(int4), cudaMemcpyHostToDevice));
        view_pair_tile.ensure(worlds);
        CK(cudaMemcpy(view_pair_tile.p, pair_first.data(), pair_first.size() * sizeof(int), cudaMemcpyHostToDevice));
        world_first.ensure(worlds + 1);
        CK(cudaMemcpy(world_first.p, world_first_host.data(), (worlds + 1) * sizeof(int), cudaMemcpyHostToDevice));
        params.world_first = world_first.p;
    }
    if (n == 0) {
        CK(cudaEventRecord(ev_done, stream));
        wait(ev_done, timeout);
        return;
    }

    // The meshes' trees, built once on the host (src/mesh_build.cpp:91-157), and the slots' tables.
    const BuiltMeshes built = build_meshes(s, true);
    auto upload = [&](auto &buf, const auto &vec) {
        using T = std::remove_pointer_t<decltype(buf.p)>;
        const size_t bytes = vec.size() * sizeof(typename std::decay_t<decltype(vec)>::value_type);
        buf.ensure(bytes / sizeof(T));
        CK(cudaMemcpy(buf.p, vec.data(), bytes, cudaMemcpyHostToDevice));
    };
    upload(blas, built.nodes);
    upload(tris, built.triangles);
    if (!built.attributes.empty()) upload(attrs, built.attributes);
    upload(tri_index, built.triangle_index);
    // Each mesh's triangles are packed together, from its first packed triangle on (in leaf order), so a
    // mesh-local triangle index finds its packed triangle through one table.
    std::vector<int> mesh_base(s.mesh_count + 1, 0);
    for (int m = 0; m < s.mesh_count; ++m) mesh_base[m + 1] = mesh_base[m] + s.meshes[m].index_count / 3;
    std::vector<int> local_to_packed(built.triangle_index.size());
    for (int m = 0; m < s.mesh_count; ++m)
        for (int p = mesh_base[m]; p < mesh_base[m + 1]; ++p) local_to_packed[mesh_base[m] + built.triangle_index[p]] = p;
    upload(tri_of_local, local_to_packed);
    // The slot tables: one entry per slot of a world, or per instance when worlds are uneven.
    const int slots = uneven ? static_cast<int>(n) : per_world;
    std::vector<int> root_of_slot(slots);
    std::vector<float> bounds_of_slot(6 * static_cast<size_t>(slots));
    std::vector<DevMaterial> material_of_slot(slots);
    for (int i = 0; i < slots; ++i) {
        const int mesh = s.instances[i].mesh;
        root_of_slot[i] = built.roots[mesh];
        std::copy(built.bounds.begin() + 6 * mesh, built.bounds.begin() + 6 * mesh + 6, bounds_of_slot.begin() + 6 * i);
        material_of_slot[i] = dev_material(s.instances[i].material);
    }
    upload(slot_blas_root, root_of_slot);
    std::vector<float4> hull_of_mesh(s.mesh_count), hull_of_slot(slots);
    for (int m = 0; m < s.mesh_count; ++m) {
        const std::array<float, 4> h = mesh_hull(s.meshes[m]);
        hull_of_mesh[m] = make_float4(h[0], h[1], h[2], h[3]);
    }
    for (int i = 0; i < slots; ++i) hull_of_slot[i] = hull_of_mesh[s.instances[i].mesh];
    upload(slot_hull, hull_of_slot);
    std::vector<float4> sphere_of_mesh(s.mesh_count), sphere_of_slot(slots);
    for (int m = 0; m < s.mesh_count; ++m) {
        const std::array<float, 4> b = mesh_sphere(s.meshes[m]);
        sphere_of_mesh[m] = make_float4(b[0], b[1], b[2], b[3]);
    }
    for (int i = 0; i < slots; ++i) sphere_of_slot[i] = sphere_of_mesh[s.instances[i].mesh];
    upload(slot_sphere, sphere_of_slot);
    std::vector<int> tri_base_of_slot(slots);
    for (int i = 0; i < slots; ++i) tri_base_of_slot[i] = mesh_base[s.instances[i].mesh];
    upload(slot_tri_base, tri_base_of_slot);
    upload(blas_pairs, built.pairs);
    std::vector<int2> root_ref_of_slot(slots);
    for (int i = 0; i < slots; ++i) {
        const int mesh = s.instances[i].mesh;
        root_ref_of_slot[i] = make_int2(built.root_refs[2 * mesh], built.root_refs[2 * mesh + 1]);
    }
    upload(slot_root, root_ref_of_slot);
    // What a device rebuild of a mesh's tree needs: its place in the packed arrays, its indices, its normals.
    {
        std::vector<uint32_t> all_indices;
        std::vector<float> all_normals;
        for (int m = 0; m < s.mesh_count; ++m) {
            const ngb_mesh &mesh = s.meshes[m];
            mesh_node_base.push_back(built.roots[m]);
            mesh_tri_base.push_back(mesh_base[m]);
            mesh_tris.push_back(mesh.index_count / 3);
            mesh_verts.push_back(mesh.vertex_count);
            mesh_nodes.push_back(built.node_counts[m]);
            mesh_index_at.push_back(static_cast<int>(all_indices.size()));
            all_indices.insert(all_indices.end(), mesh.indices, mesh.indices + mesh.index_count);
            mesh_normal_at.push_back(mesh.normals ? static_cast<int>(all_normals.size()) : -1);
            if (mesh.normals) all_normals.insert(all_normals.end(), mesh.normals, mesh.normals + 3 * static_cast<size_t>(mesh.vertex_count));
        }
        if (!all_indices.empty()) upload(mesh_indices, all_indices);
        if (!all_normals.empty()) upload(mesh_normals, all_normals);
        std::vector<int> mesh_of_slot(slots);
        for (int i = 0; i < slots; ++i) mesh_of_slot[i] = s.instances[i].mesh;
        if (slots > 0) upload(slot_mesh, mesh_of_slot);
        slot_mesh_host = mesh_of_slot;
    }
    tlas_pairs.ensure(4 * std::max<long long>(n - 1, 1));
    upload(slot_bounds, bounds_of_slot);
    upload(slot_material, material_of_slot);
    matrices.ensure(12 * n);
    inst.ensure(4 * n);
    tlas.ensure(2 * (2 * n - 1));
    keys.ensure(n);
    sorted_ids.ensure(n);
    roots.ensure(worlds);
    parent.ensure(2 * n - 1);
    leaf_of.ensure(n);
    arrivals.ensure(std::max<long long>(n - 1, 1));
    CK(cudaMemset(parent.p, 0xFF, (2 * n - 1) * sizeof(int)));
    CK(cudaMemset(arrivals.p, 0, arrivals.n * sizeof(int)));
    params.tlas = tlas.p;
    params.roots = roots.p;
    params.inst = inst.p;
    params.blas = blas.p;
    params.tris = tris.p;
    params.attrs = built.attributes.empty() ? nullptr : attrs.p;
    params.tri_index = tri_index.p;
    params.slot_material = slot_material.p;
    params.blas_node_count = static_cast<int>(built.nodes.size() / 8);
    params.blas_pairs = blas_pairs.p;
    params.tlas_pairs = tlas_pairs.p;
    params.slot_root = slot_root.p;
    params.slot_bounds = slot_bounds.p;
    params.tlas_internal = static_cast<int>(n - 1);
    params.slot_hull = slot_hull.p;
    params.slot_sphere = slot_sphere.p;
    params.leaf_of = leaf_of.p;

    // Every world starts with the transforms the instances were given (src/cuda_backend.cu:765-770).
    std::vector<float> initial(12 * n);
    if (uneven) {
        for (long long g = 0; g < n; ++g) std::memcpy(&initial[12 * g], s.instances[g].transform, 48);
    } else {
        for (int w = 0; w < worlds; ++w)
            for (int i = 0; i < per_world; ++i)
                std::memcpy(&initial[12 * (static_cast<size_t>(w) * per_world + i)], s.instances[i].transform, 48);
    }
    CK(cudaMemcpy(matrices.p, initial.data(), initial.size() * sizeof(float), cudaMemcpyHostToDevice));
    build(matrices.p, 0, nullptr);
    CK(cudaEventRecord(ev_done, stream));
    wait(ev_done, timeout);
}

// Frees everything; safe on a renderer whose construction stopped part way, and twice.
void Renderer::teardown() {
    // Must not throw; errors after a sticky fault are ignored. Nothing to free before the first CUDA call.
    if (!cuda_touched) return;
    int previous = -1;
    cudaGetDevice(&previous);
    if (previous != device) cudaSetDevice(device);
    if (own_stream) cudaStreamSynchronize(own_stream);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    for (cudaEvent_t &e : ev_stage) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    if (ev_done) cudaEventDestroy(ev_done);
    if (host_error) cudaFreeHost(host_error);
    if (host_count) cudaFreeHost(host_count);
    if (own_stream) cudaStreamDestroy(own_stream);
    ev_start = ev_stop = ev_done = nullptr;
    host_error = host_count = nullptr;
    own_stream = nullptr;
    // The DevBufs free themselves; the device must be current while they do, so release them here.
    blas.release(), tris.release(), attrs.release(), tri_index.release(), slot_blas_root.release();
    tri_of_local.release(), slot_tri_base.release();
    slot_bounds.release(), slot_material.release(), matrices.release(), inst.release(), tlas.release();
    keys.release(), sorted_ids.release(), roots.release(), parent.release(), arrivals.release();
    body_of_instance.release(), local_pose.release(), local_scale.release(), body_poses.release();
    geom_of_instance.release(), geom_scale.release(), geom_xpos.release(), geom_xmat.release();
    mesh_indices.release(), mesh_normals.release(), mesh_stage.release(), slot_mesh.release();
    mb_box.release(), mb_centre.release(), mb_node_box.release(), mb_order.release(), mb_lpos.release();
    mb_rpos.release(), mb_begin.release(), mb_end.release(), mb_left.release(), mb_depth.release();
    mb_index.release(), mb_counter.release(), mb_starts.release(), mb_top.release(), mb_prefix.release();
    mb_level_count.release();
    blas_pairs.release(), tlas_pairs.release(), slot_root.release(), work_counter.release();
    large_aabb.release(), large_bounds.release(), large_ids_a.release(), large_ids_b.release();
    large_keys_a.release(), large_keys_b.release(), large_counts.release();
    pic_hit.release(), shadow_o.release(), shadow_d.release(), pic_code.release(), shadow_self.release();
    view_order.release(), view_bound.release();
    leaf_of.release(), slot_hull.release(), slot_sphere.release();
    camera_basis.release(), srgb_table.release();
    cameras.release(), ray_origins.release(), ray_directions.release(), out_rgb.release(), out_depth.release();
    out_normal.release(), out_id.release(), ray_distance.release(), ray_normal.release(), ray_id.release();
    hit_instance.release(), hit_triangle.release(), hit_u.release(), hit_v.release(), error_flag.release();
    world_first.release(), view_info.release(), view_pair_tile.release();
    view_accum.release(), view_radiance.release(), view_argb.release();
    if (previous >= 0 && previous != device) cudaSetDevice(previous);
}

// Waits for an event with a limit: polls, and gives up with NGB_TIMEOUT after `seconds`.
void Renderer::wait(cudaEvent_t ev, double seconds) {
    const auto start = std::chrono::steady_clock::now();
    for (int spin = 0;; ++spin) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return;
        if (e != cudaErrorNotReady) CK(e);
        const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        if (waited > seconds)
            throw Timeout("the GPU work did not finish within " + std::to_string(seconds) + " seconds");
        if (spin > 1000) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// Called after every launch: brings the device's error flag back with the work and, when synchronous,
// waits for both.
// The last launch's GPU times, once its events have completed.
void Renderer::read_timing() {
    if (!timing_pending) return;
    CK(cudaEventElapsedTime(&kernel_ms, ev_start, ev_stop));
    if (stages == 3) {
        CK(cudaEventElapsedTime(&stage_ms[0], ev_start, ev_stage[0]));
        CK(cudaEventElapsedTime(&stage_ms[1], ev_stage[0], ev_stage[1]));
        CK(cudaEventElapsedTime(&stage_ms[2], ev_stage[1], ev_stop));
    } else {
        stage_ms[0] = kernel_ms;
    }
    timing_pending = false;
}

// Queues the copy of the device error flag to host_error, for a wait that follows.
void Renderer::queue_error_read() {
    CK(cudaMemcpyAsync(host_error, error_flag.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
}

void Renderer::finish() {
    // Stream-ordered calls and graph captures queue no copy of the flag: a device-to-host copy in the stream
    // waits behind every such copy the caller has on the copy engine (the last step's images going out while
    // this step renders) and holds back the launches queued after it. ngb_synchronize reads the flag.
    if (capturing() || !synchronous) return;
    queue_error_read();
    CK(cudaEventRecord(ev_done, stream));
    wait(ev_done, timeout);
    read_timing();
    if (*host_error) throw CudaFailure(-1, device_error_message(*host_error));
}

// Queues the tree build of every world: from matrices in device memory (compose 0), or composed from body
// poses (1: poses) or geom poses (2: poses are the positions, xmat the rotations).
void Renderer::build(const float *matrices_in, int compose, const float *poses, const float *xmat) {
    BuildArgs a{};
    a.worlds = worlds;
    a.per_world = per_world;
    a.n = n;
    a.compose = compose;
    a.matrices_in = matrices_in;
    a.body_poses = compose == 1 ? poses : nullptr;
    a.body_of_instance = body_of_instance.p;
    a.local_pose = local_pose.p;
    a.local_scale = local_scale.p;
    a.bodies_per_world = bodies_per_world;
    a.geom_xpos = compose == 2 ? poses : nullptr;
    a.geom_xmat = xmat;
    a.geom_of_instance = geom_of_instance.p;
    a.geom_scale = geom_scale.p;
    a.geoms_per_world = geoms_per_world;
    // Composed matrices, and matrices given in the caller's device memory, are kept for inspection.
    a.matrices_out = (compose || matrices_in != matrices.p) ? matrices.p : nullptr;
    a.slot_bounds = slot_bounds.p;
    a.slot_blas_root = slot_blas_root.p;
    a.inst = inst.p;
    a.keys = keys.p;
    a.sorted_ids = sorted_ids.p;
    a.tlas = tlas.p;
    a.roots = roots.p;
    a.parent = parent.p;
    a.arrivals = arrivals.p;
    a.error_flag = error_flag.p;
    a.tlas_pairs = tlas_pairs.p;
    a.world_first = uneven ? world_first.p : nullptr;
    a.leaf_of = leaf_of.p;
    if (use_large_build()) {
        LargeBuildScratch t{};
        t.aabb = large_aabb.ensure(2 * n);
        t.bounds = large_bounds.ensure(6 * static_cast<size_t>(worlds));
        t.keys_a = large_keys_a.ensure(n);
        t.keys_b = large_keys_b.ensure(n);
        t.ids_a = large_ids_a.ensure(n);
        t.ids_b = large_ids_b.ensure(n);
        t.counts = large_counts.ensure(256 * static_cast<size_t>(large_sort_blocks(n)));
        CK(launch_build_large(a, t, stream));
    } else {
        CK(launch_build_worlds(a, stream));
    }
}

// src/batch.cpp:91-109 and src/cuda_backend.cu:457-469.
void Renderer::set_instance_transforms(const float *m, int memory) {
    Range range("ngb set_instance_transforms");
    require(memory == NGB_MEMORY_HOST || memory == NGB_MEMORY_DEVICE, "memory must be NGB_MEMORY_HOST or NGB_MEMORY_DEVICE");
    if (n == 0) return;
    require(m != nullptr, "matrices must not be null");
    if (memory == NGB_MEMORY_HOST) {
        for (long long g = 0; g < n; ++g)
            if (!transform_ok(m + 12 * g)) {
                const int w = world_of_instance(g);
                const long long first = uneven ? world_first_host[w] : static_cast<long long>(w) * per_world;
                check_transform(m + 12 * g, "world " + std::to_string(w) + " instance " + std::to_string(g - first) +
                    " transform");
            }
        CK(cudaMemcpyAsync(matrices.p, m, static_cast<size_t>(n) * 12 * sizeof(float), cudaMemcpyHostToDevice, stream));
        build(matrices.p, 0, nullptr);
    } else {
        build(m, 0, nullptr);
    }
    finish();
}

// src/batch.cpp:111-129 and src/cuda_backend.cu:472-491.
void Renderer::bind_bodies(int bpw, const int32_t *boi, const float *lp, const float *sc) {
    require(!uneven, "worlds of uneven sizes take instance matrices (set_instance_transforms), not body poses");
    const int P = per_world;
    require(bpw >= 0, "bodies_per_world must be 0 or more");
    require(P == 0 || (boi != nullptr && lp != nullptr && sc != nullptr),
        "a body binding needs one body index, 7 pose floats and 3 scale floats for each of the " + std::to_string(P) +
        " instances of a world");
    for (int i = 0; i < P; ++i) {
        const int b = boi[i];
        require(b >= -1 && b < bpw, "instance " + std::to_string(i) + " is on body " + std::to_string(b) +
            ", but there are " + std::to_string(bpw) + " bodies per world");
        require(all_finite(lp + 7 * i, 7) && quaternion_is_usable(lp + 7 * i + 3),
            "instance " + std::to_string(i) + " has a pose with a NaN or infinite value, or a zero quaternion");
        require(all_finite(sc + 3 * i, 3), "instance " + std::to_string(i) + " has a scale with a NaN or infinite value");
    }
    require(static_cast<long long>(worlds) * bpw * 7 <= INT32_MAX, "too many bodies");
    if (P > 0) {
        body_of_instance.ensure(P);
        local_pose.ensure(7 * static_cast<size_t>(P));
        local_scale.ensure(3 * static_cast<size_t>(P));
        CK(cudaMemcpyAsync(body_of_instance.p, boi, P * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(local_pose.p, lp, 7 * P * sizeof(float), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(local_scale.p, sc, 3 * P * sizeof(float), cudaMemcpyHostToDevice, stream));
        body_poses.ensure(7 * static_cast<size_t>(worlds) * bpw);
        CK(cudaEventRecord(ev_done, stream));
        wait(ev_done, timeout);  // the host arrays are the caller's; the copies must be done
    }
    bodies_per_world = bpw;
    bound = true;
    geoms_bound = false;
}

// src/batch.cpp:131-144 and src/cuda_backend.cu:493-507.
void Renderer::set_body_poses(const float *poses, int memory) {
    Range range("ngb set_body_poses");
    require(bound, "set_body_poses needs bind_bodies to be called first");
    require(memory == NGB_MEMORY_HOST || memory == NGB_MEMORY_DEVICE, "memory must be NGB_MEMORY_HOST or NGB_MEMORY_DEVICE");
    const size_t bodies = static_cast<size_t>(worlds) * bodies_per_world;
    require(bodies == 0 || poses != nullptr, "body_poses must not be null");
    if (memory == NGB_MEMORY_HOST)
        for (size_t b = 0; b < bodies; ++b)
            require(all_finite(poses + 7 * b, 7) && quaternion_is_usable(poses + 7 * b + 3),
                "body " + std::to_string(b) + " has a NaN or infinite value, or a zero quaternion");
    if (per_world == 0) return;
    const float *src = poses;
    if (memory == NGB_MEMORY_HOST && bodies > 0) {
        CK(cudaMemcpyAsync(body_poses.p, poses, bodies * 7 * sizeof(float), cudaMemcpyHostToDevice, stream));
        src = body_poses.p;
    }
    build(nullptr, 1, src);
    finish();
}

// The geom list and scales of MJWarpBatchRenderer (python/neraulgraphics/mujoco.py:199-243), checked as a
// body binding is.
void Renderer::bind_geoms(int gpw, const int32_t *goi, const float *sc) {
    require(!uneven, "worlds of uneven sizes take instance matrices (set_instance_transforms), not geom poses");
    const int P = per_world;
    require(gpw >= 0, "geoms_per_world must be 0 or more");
    require(P == 0 || (goi != nullptr && sc != nullptr),
        "a geom binding needs one geom index and 3 scale floats for each of the " + std::to_string(P) +
        " instances of a world");
    for (int i = 0; i < P; ++i) {
        const int g = goi[i];
        require(g >= 0 && g < gpw, "instance " + std::to_string(i) + " is on geom " + std::to_string(g) +
            ", but there are " + std::to_string(gpw) + " geoms per world");
        require(all_finite(sc + 3 * i, 3), "instance " + std::to_string(i) + " has a scale with a NaN or infinite value");
    }
    require(static_cast<long long>(worlds) * gpw * 9 <= INT32_MAX, "too many geoms");
    if (P > 0) {
        geom_of_instance.ensure(P);
        geom_scale.ensure(3 * static_cast<size_t>(P));
        CK(cudaMemcpyAsync(geom_of_instance.p, goi, P * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(geom_scale.p, sc, 3 * P * sizeof(float), cudaMemcpyHostToDevice, stream));
        geom_xpos.ensure(3 * static_cast<size_t>(worlds) * gpw);
        geom_xmat.ensure(9 * static_cast<size_t>(worlds) * gpw);
        CK(cudaEventRecord(ev_done, stream));
        wait(ev_done, timeout);  // the host arrays are the caller's; the copies must be done
    }
    geoms_per_world = gpw;
    geoms_bound = true;
    bound = false;
}

// MJWarpBatchRenderer.update (python/neraulgraphics/mujoco.py:304-314): compose and build in one launch.
void Renderer::set_geom_poses(const float *xpos, const float *xmat, int memory) {
    Range range("ngb set_geom_poses");
    require(geoms_bound, "set_geom_poses needs bind_geoms to be called first");
    require(memory == NGB_MEMORY_HOST || memory == NGB_MEMORY_DEVICE, "memory must be NGB_MEMORY_HOST or NGB_MEMORY_DEVICE");
    const size_t geoms = static_cast<size_t>(worlds) * geoms_per_world;
    require(geoms == 0 || (xpos != nullptr && xmat != nullptr), "geom_xpos and geom_xmat must not be null");
    if (memory == NGB_MEMORY_HOST)
        for (size_t g = 0; g < geoms; ++g)
            require(all_finite(xpos + 3 * g, 3) && all_finite(xmat + 9 * g, 9),
                "geom " + std::to_string(g) + " has a NaN or infinite position or rotation");
    if (per_world == 0) return;
    const float *p = xpos, *r = xmat;
    if (memory == NGB_MEMORY_HOST && geoms > 0) {
        CK(cudaMemcpyAsync(geom_xpos.p, xpos, geoms * 3 * sizeof(float), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(geom_xmat.p, xmat, geoms * 9 * sizeof(float), cudaMemcpyHostToDevice, stream));
        p = geom_xpos.p;
        r = geom_xmat.p;
    }
    build(nullptr, 2, p, r);
    finish();
}

// New vertex positions for one mesh: its tree rebuilt on the device as the host builds it at creation
// (src/bvh.cpp:46-174, src/mesh_build.cpp:91-157), then every world's instance tree from the current
// transforms, whose boxes hold the mesh's new box.
void Renderer::update_mesh(int mesh, const float *vertices, const float *normals, int memory) {
    Range range("ngb update_mesh");
    require(mesh >= 0 && mesh < static_cast<int>(mesh_tris.size()),
        "mesh " + std::to_string(mesh) + " does not exist: there are " + std::to_string(mesh_tris.size()) + " meshes");
    require(memory == NGB_MEMORY_HOST || memory == NGB_MEMORY_DEVICE, "memory must be NGB_MEMORY_HOST or NGB_MEMORY_DEVICE");
    require(vertices != nullptr, "vertices must not be null");
    require(normals == nullptr || mesh_normal_at[mesh] >= 0,
        "mesh " + std::to_string(mesh) + " was made without vertex normals, so update_mesh cannot give it some");
    const int V = mesh_verts[mesh], T = mesh_tris[mesh];
    const std::string name = "mesh " + std::to_string(mesh);
    if (memory == NGB_MEMORY_HOST) {
        for (int i = 0; i < V; ++i)
            require(all_finite(vertices + 3 * static_cast<size_t>(i), 3), name + " vertex " + std::to_string(i) +
                " has a NaN or infinite value");
        if (normals)
            for (int i = 0; i < V; ++i)
                require(all_finite(normals + 3 * static_cast<size_t>(i), 3), name + " normal " + std::to_string(i) +
                    " has a NaN or infinite value");
    }
    const cudaMemcpyKind kind = memory == NGB_MEMORY_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const float *dv = vertices;
    if (memory == NGB_MEMORY_HOST) {
        mesh_stage.ensure(3 * static_cast<size_t>(V));
        CK(cudaMemcpyAsync(mesh_stage.p, vertices, 3 * static_cast<size_t>(V) * sizeof(float), kind, stream));
        dv = mesh_stage.p;
    }
    float *kept_normals = mesh_normal_at[mesh] >= 0 ? mesh_normals.p + mesh_normal_at[mesh] : nullptr;
    if (normals) CK(cudaMemcpyAsync(kept_normals, normals, 3 * static_cast<size_t>(V) * sizeof(float), kind, stream));

    MeshBuildScratch t{};
    t.box = mb_box.ensure(6 * static_cast<size_t>(T));
    t.centre = mb_centre.ensure(3 * static_cast<size_t>(T));
    t.order = mb_order.ensure(T);
    t.lpos = mb_lpos.ensure(T);
    t.rpos = mb_rpos.ensure(T);
    const size_t cap = 2 * static_cast<size_t>(T) - 1;
    t.node_box = mb_node_box.ensure(6 * cap);
    t.begin = mb_begin.ensure(cap);
    t.end = mb_end.ensure(cap);
    t.left = mb_left.ensure(cap);
    t.depth = mb_depth.ensure(cap);
    t.index = mb_index.ensure(cap);
    t.counter = mb_counter.ensure(1);
    t.level_count = mb_level_count.ensure(MESH_LEVELS + 1);
    t.starts = mb_starts.ensure(T);
    t.top = mb_top.ensure(T);
    t.prefix = mb_prefix.ensure(T);
    MeshBuildArgs a{};
    a.vertices = dv;
    a.normals = kept_normals;
    a.indices = mesh_indices.p + mesh_index_at[mesh];
    a.triangles = T;
    a.node_base = mesh_node_base[mesh];
    a.tri_base = mesh_tri_base[mesh];
    a.blas = blas.p;
    a.pairs = blas_pairs.p;
    a.tris = tris.p;
    a.attrs = attrs.p;
    a.tri_index = tri_index.p;
    a.tri_of_local = tri_of_local.p;
    // One cooperative launch builds and packs the tree (clearing the mesh's whole node run first, so nodes past
    // the new tree's last are zero, as at creation); its node count comes back for inspection.
    CK(launch_mesh_build(a, t, slot_mesh.p, slot_mesh.p ? static_cast<int>(slot_mesh.n) : 0, mesh, slot_root.p,
        slot_bounds.p, slot_hull.p, stream));
    // The new shape has no bounding sphere: its slots' walks go without the sphere test.
    static const float no_sphere = -1.0f;
    for (size_t i = 0; i < slot_mesh_host.size(); ++i)
        if (slot_mesh_host[i] == mesh)
            CK(cudaMemcpyAsync(reinterpret_cast<float *>(slot_sphere.p + i) + 3, &no_sphere, sizeof(float),
                cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(host_count, t.counter, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaEventRecord(ev_done, stream));
    wait(ev_done, timeout);
    require(*host_count >= 1 && static_cast<size_t>(*host_count) <= cap, name + ": the tree rebuild went wrong");
    mesh_nodes[mesh] = *host_count;
    if (n > 0) build(matrices.p, 0, nullptr);
    finish();
}

// src/batch.cpp:146-162: every argument check, in the reference's order.
void Renderer::check_render(const float *cams, float fov, int spp, unsigned outputs, int frame, int memory) {
    constexpr unsigned ALL = NGB_OUTPUT_RGB | NGB_OUTPUT_DEPTH | NGB_OUTPUT_NORMAL | NGB_OUTPUT_OBJECT_ID;
    require(outputs != 0, "render needs at least one output");
    require((outputs & ~ALL) == 0, "unknown output bits in " + std::to_string(outputs));
    require(spp >= 1, "samples_per_pixel must be 1 or more, got " + std::to_string(spp));
    require(frame >= 0, "frame must be 0 or more, got " + std::to_string(frame));
    require(fov > 0.0f && fov < 3.14159265f, "fov must be between 0 and pi radians, got " + fstr(fov));
    require(memory == NGB_MEMORY_HOST || memory == NGB_MEMORY_DEVICE, "memory must be NGB_MEMORY_HOST or NGB_MEMORY_DEVICE");
    require(cams != nullptr, "camera_matrices must not be null");
    if (memory == NGB_MEMORY_HOST)
        require(all_finite(cams, 12 * static_cast<size_t>(worlds) * cpw), "a camera has a NaN or infinite value");
}

// The lights as the kernels read them (the reference's to_device: src/device_scene.h:265-272).
void Renderer::put_lights(const ngb_light *lights, int count) {
    for (int i = 0; i < count; ++i) {
        const ngb_light &l = lights[i];
        float dx = l.direction.x, dy = l.direction.y, dz = l.direction.z;
        const float nn = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (nn > 0.0f) {
            dx = dx / nn;
            dy = dy / nn;
            dz = dz / nn;
        } else {
            dx = 0.0f;
            dy = 0.0f;
            dz = -1.0f;
        }
        const bool spot = l.spot_angle > 0.0f;
        params.lights[i] = DevLight{make_float3(l.position.x, l.position.y, l.position.z), l.intensity, l.radius, l.falloff,
            make_float3(dx, dy, dz), spot ? std::cos(l.spot_angle) : -2.0f,
            spot ? std::cos(l.spot_angle * (1.0f - l.spot_softness)) : -2.0f, make_float3(l.color.x, l.color.y, l.color.z)};
    }
    params.light_count = count;
}

// src/renderer.cpp:104-108, 174-182 and src/validate.cpp:82-89: a single-view render's checks.
void Renderer::check_view(const ngb_camera *c, int frame, int spp) {
    require(worlds == 1 && cpw == 1 && !uneven,
        "a view render needs a renderer of one world seen by one camera (world_count 1, cameras_per_world 1)");
    require(c != nullptr, "camera must not be null");
    require(frame >= 0, "frame must be 0 or more, got " + std::to_string(frame));
    require(spp >= 1, "samples_per_frame must be 1 or more, got " + std::to_string(spp));
    const float v[14] = {c->position.x, c->position.y, c->position.z, c->right.x, c->right.y, c->right.z, c->up.x,
        c->up.y, c->up.z, c->forward.x, c->forward.y, c->forward.z, c->fov_scale, c->aspect};
    require(all_finite(v, 14), "camera has a NaN or infinite value (is its target on the view axis, or up parallel to it?)");
}

void Renderer::render(const float *cams, float fov, int spp, unsigned outputs, int frame, int memory, uint8_t *rgb,
    float *depth, float *normal, int32_t *ids, const ngb_camera *view) {
    Range range(view ? "ngb render_view" : "ngb render");
    const int views = worlds * cpw;
    const float *cam = cams;
    if (view) {
        cam = nullptr;
    } else if (memory == NGB_MEMORY_HOST) {
        cameras.ensure(12 * static_cast<size_t>(views));
        CK(cudaMemcpyAsync(cameras.p, cams, 12 * static_cast<size_t>(views) * sizeof(float), cudaMemcpyHostToDevice, stream));
        cam = cameras.p;
    }
    RenderArgs a{};
    a.cameras = cam;
    a.fov_scale = std::tan(fov * 0.5f);  // tanf on the host, as the reference's CPU backend computes it
    a.aspect = uneven ? 1.0f : static_cast<float>(width) / static_cast<float>(height);
    if (view) {
        // The camera as the caller gave it (src/cuda_backend.cu:651-652 passes it to the kernel unchanged).
        a.fov_scale = view->fov_scale;
        a.aspect = view->aspect;
        const float4 basis[3] = {make_float4(view->position.x, view->position.y, view->position.z, view->right.x),
            make_float4(view->right.y, view->right.z, view->up.x, view->up.y),
            make_float4(view->up.z, view->forward.x, view->forward.y, view->forward.z)};
        a.camera_basis = camera_basis.ensure(3);
        CK(cudaMemcpyAsync(a.camera_basis, basis, sizeof(basis), cudaMemcpyHostToDevice, stream));
        a.basis_given = 1;
    }
    a.width = width;
    a.height = height;
    a.row_first = band_first;
    a.rows = rows();
    a.cameras_per_world = cpw;
    a.views = views;
    a.frame = frame;
    a.spp = spp;
    a.rgb = (outputs & NGB_OUTPUT_RGB) ? rgb : nullptr;
    a.depth = (outputs & NGB_OUTPUT_DEPTH) ? depth : nullptr;
    a.normal = (outputs & NGB_OUTPUT_NORMAL) ? normal : nullptr;
    a.object_id = (outputs & NGB_OUTPUT_OBJECT_ID) ? ids : nullptr;
    if (record_hits && (outputs & (NGB_OUTPUT_DEPTH | NGB_OUTPUT_NORMAL | NGB_OUTPUT_OBJECT_ID))) {
        if (ext_instance) {
            a.hit_instance = ext_instance;
            a.hit_triangle = ext_triangle;
            a.hit_u = ext_u;
            a.hit_v = ext_v;
        } else {
            a.hit_instance = hit_instance.ensure(pixels());
            a.hit_triangle = hit_triangle.ensure(pixels());
            a.hit_u = hit_u.ensure(pixels());
            a.hit_v = hit_v.ensure(pixels());
        }
    }
    a.error_flag = error_flag.p;
    // The persistent and tile kernels cover one sample per pixel, at most one light and no bounces; everything
    // else takes the per-pixel kernel, which runs trace in full. Automatic: the tile kernels (candidate lists
    // for worlds of at most TILE_MAX_INSTANCES instances, a packet walk of the world tree above).
    const bool persistent_ok = spp == 1 && params.light_count <= 1 && !reflective;
    // A view render's picture is a running average of radiance, which the tile and per-pixel kernels hand over.
    const bool tiles = persistent_ok && (uneven || kernel_choice == 3 || kernel_choice == 0 || (view && kernel_choice == 2));
    const bool persistent = !view && !tiles && persistent_ok && (kernel_choice == 0 || kernel_choice == 2);
    if (view && a.rgb) {
        a.radiance = view_radiance.ensure(pixels());
        if (view_accum.n < pixels()) {
            view_accum.ensure(pixels());
            CK(cudaMemsetAsync(view_accum.p, 0, pixels() * sizeof(float4), stream));
        }
        view_argb.ensure(pixels());
    }
    require(!uneven || tiles, "worlds of uneven sizes render with one sample per pixel, at most one light and no "
        "reflective material");
    // Inside a CUDA graph capture the timing events would be graph nodes whose times cannot be read: the
    // render is then not timed (last_kernel_ms keeps the previous figure).
    const bool timed = !capturing();
    if (timed) CK(cudaEventRecord(ev_start, stream));
    if (tiles) {
        a.camera_basis = camera_basis.ensure(3 * static_cast<size_t>(views));
        if (per_world > 0 && per_world <= TILE_MAX_INSTANCES) {
            a.view_order = view_order.ensure(static_cast<size_t>(views) * per_world);
            a.view_bound = view_bound.ensure(static_cast<size_t>(views) * per_world);
            a.order_stride = per_world;
        }
        if (uneven) {
            a.view_info = view_info.p;
            a.total_pixels = total_pixels;
            a.total_tiles = total_tiles;
            a.view_pair_tile = view_pair_tile.p;
            a.total_pair_tiles = total_pair_tiles;
        }
        if (a.rgb) {
            a.pic_hit = pic_hit.ensure(pixels());
            a.pic_code = pic_code.ensure(pixels());
            a.shadow_o = shadow_o.ensure(pixels());
            a.shadow_d = shadow_d.ensure(pixels());
            a.shadow_self = shadow_self.ensure(pixels());
        }
        CK(launch_render_tiles(params, a, reinterpret_cast<int *>(work_counter.p), tile_tuning, stream,
            timed ? ev_stage[0] : nullptr, timed ? ev_stage[1] : nullptr));
        stages = 3;
    } else if (persistent) {
        a.camera_basis = camera_basis.ensure(3 * static_cast<size_t>(views));
        CK(launch_render_persistent(params, a, reinterpret_cast<int *>(work_counter.p), tuning, stream));
        stages = 1;
    } else {
        CK(launch_render(params, a, stream));
        stages = 1;
    }
    if (a.radiance)
        CK(launch_accumulate(a.radiance, view_accum.p, frame, static_cast<long long>(pixels()), srgb_table.p,
            view_argb.p, a.rgb, stream));
    if (timed) {
        CK(cudaEventRecord(ev_stop, stream));
        timing_pending = true;
    }
    finish();
}

// src/batch.cpp:180-192 and src/cuda_backend.cu:547-585.
void Renderer::cast_rays(const float *o, const float *d, int rays_per_world, float max_distance, int memory,
    ngb_ray_hits *out, float *distance, float *normal, int32_t *ids) {
    Range range("ngb cast_rays");
    require(rays_per_world >= 0, "rays_per_world must be 0 or more, got " + std::to_string(rays_per_world));
    const long long count = static_cast<long long>(rays_per_world) * worlds;
    require(count <= INT32_MAX / 3, "too many rays: " + std::to_string(count));
    require(count == 0 || (o != nullptr && d != nullptr), "ray origins and directions must not be null");
    require(max_distance > 0.0f, "max_distance must be positive, got " + fstr(max_distance));
    require(memory == NGB_MEMORY_HOST || memory == NGB_MEMORY_DEVICE, "memory must be NGB_MEMORY_HOST or NGB_MEMORY_DEVICE");
    if (memory == NGB_MEMORY_HOST) require(all_finite(o, static_cast<size_t>(count) * 3), "a ray origin has a NaN or infinite value");
    *out = ngb_ray_hits{NGB_MEMORY_DEVICE, device, static_cast<int32_t>(count), nullptr, nullptr, nullptr};
    if (count == 0) return;
    const float *po = o, *pd = d;
    if (memory == NGB_MEMORY_HOST) {
        ray_origins.ensure(3 * count);
        ray_directions.ensure(3 * count);
        CK(cudaMemcpyAsync(ray_origins.p, o, 3 * count * sizeof(float), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(ray_directions.p, d, 3 * count * sizeof(float), cudaMemcpyHostToDevice, stream));
        po = ray_origins.p;
        pd = ray_directions.p;
    }
    RayArgs a{};
    a.origins = po;
    a.directions = pd;
    a.max_distance = max_distance;
    a.rays_per_world = rays_per_world;
    a.count = static_cast<int>(count);
    a.distance = distance ? distance : ray_distance.ensure(count);
    a.normal = normal ? normal : ray_normal.ensure(3 * count);
    a.object_id = ids ? ids : ray_id.ensure(count);
    a.error_flag = error_flag.p;
    const bool timed = !capturing();
    if (timed) CK(cudaEventRecord(ev_start, stream));
    // Automatic: warp packets for worlds above TILE_MAX_INSTANCES (a large world's rays walk long and alike: 0.43
    // against 0.58 ms for a 64 x 2048 LiDAR sweep of 100,000 instances), else the persistent kernel's lane-refilling
    // walk; the per-thread kernel when the per-pixel kernel is chosen, the persistent one when it is; or as
    // ngb_set_ray_kernel says.
    const int mode = ray_kernel != 0 ? ray_kernel
        : kernel_choice == 1                                   ? 1
        : kernel_choice != 2 && per_world > TILE_MAX_INSTANCES ? 3
                                                               : 2;
    if (mode == 1) CK(launch_rays(params, a, stream));
    else if (mode == 3) CK(launch_rays_packets(params, a, reinterpret_cast<int *>(work_counter.p), stream));
    else CK(launch_rays_persistent(params, a, reinterpret_cast<int *>(work_counter.p),
        kernel_choice == 2 ? tuning : ray_tuning, stream));
    if (timed) {
        stages = 1;
        CK(cudaEventRecord(ev_stop, stream));
        timing_pending = true;
    }
    finish();
    out->distance = a.distance;
    out->normal = a.normal;
    out->object_id = a.object_id;
}

}  // namespace ngb

// ------------------------------------------------------------------------------------------- C ABI --

struct ngb_renderer {
    ngb::Renderer r;
    explicit ngb_renderer(const ngb_scene &s, const ngb::UnevenLayout *layout = nullptr) : r(s, layout) {}
};

namespace {

thread_local std::string g_create_error;

}  // namespace

namespace ngb {
void set_global_error(const std::string &message) { g_create_error = message; }
}  // namespace ngb

namespace {

template <class F>
int guarded(ngb_renderer *h, F &&f) {
    if (h == nullptr) {
        g_create_error = "the renderer is null (destroyed or never created)";
        return NGB_LOGIC_ERROR;
    }
    std::lock_guard<std::mutex> lock(h->r.mutex);
    try {
        ngb::DeviceGuard guard(h->r.device);
        f(h->r);
        h->r.last_error.clear();
        return NGB_OK;
    } catch (const ngb::InvalidArgument &e) {
        h->r.last_error = e.what();
        return NGB_INVALID_ARGUMENT;
    } catch (const ngb::Timeout &e) {
        h->r.last_error = e.what();
        return NGB_TIMEOUT;
    } catch (const std::bad_alloc &) {
        h->r.last_error = "out of host memory";
        return NGB_CUDA_ERROR;
    } catch (const std::exception &e) {
        h->r.last_error = e.what();
        return NGB_CUDA_ERROR;
    }
}

}  // namespace

extern "C" {

int ngb_create(const ngb_scene *scene, ngb_renderer **out) {
    if (out) *out = nullptr;
    try {
        ngb::require(scene != nullptr && out != nullptr, "scene and out must not be null");
        *out = new ngb_renderer(*scene);
        g_create_error.clear();
        return NGB_OK;
    } catch (const ngb::InvalidArgument &e) {
        g_create_error = e.what();
        return NGB_INVALID_ARGUMENT;
    } catch (const ngb::Timeout &e) {
        g_create_error = e.what();
        return NGB_TIMEOUT;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return NGB_CUDA_ERROR;
    }
}

int ngb_create_uneven(const ngb_scene *scene, const ngb_uneven_world *worlds, int32_t world_count, ngb_renderer **out) {
    if (out) *out = nullptr;
    try {
        ngb::require(scene != nullptr && out != nullptr && (worlds != nullptr || world_count == 0),
            "scene, worlds and out must not be null");
        ngb::require(world_count >= 1, "world_count must be 1 or more, got " + std::to_string(world_count));
        ngb::UnevenLayout layout;
        layout.first.assign(1, 0);
        for (int w = 0; w < world_count; ++w) {
            ngb::require(worlds[w].instance_count >= 0, "world " + std::to_string(w) + " has a negative instance count");
            layout.first.push_back(layout.first.back() + worlds[w].instance_count);
            layout.width.push_back(worlds[w].width);
            layout.height.push_back(worlds[w].height);
        }
        *out = new ngb_renderer(*scene, &layout);
        g_create_error.clear();
        return NGB_OK;
    } catch (const ngb::InvalidArgument &e) {
        g_create_error = e.what();
        return NGB_INVALID_ARGUMENT;
    } catch (const ngb::Timeout &e) {
        g_create_error = e.what();
        return NGB_TIMEOUT;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return NGB_CUDA_ERROR;
    }
}

int64_t ngb_pixel_count(const ngb_renderer *h) { return h ? static_cast<int64_t>(h->r.pixels()) : 0; }

void ngb_destroy(ngb_renderer *r) { delete r; }

const char *ngb_last_error(const ngb_renderer *r) { return r ? r->r.last_error.c_str() : g_create_error.c_str(); }

int ngb_set_instance_transforms(ngb_renderer *h, const float *m, int32_t memory) {
    return guarded(h, [&](ngb::Renderer &r) { r.set_instance_transforms(m, memory); });
}

int ngb_bind_bodies(ngb_renderer *h, int32_t bpw, const int32_t *boi, const float *lp, const float *sc) {
    return guarded(h, [&](ngb::Renderer &r) { r.bind_bodies(bpw, boi, lp, sc); });
}

int ngb_set_body_poses(ngb_renderer *h, const float *poses, int32_t memory) {
    return guarded(h, [&](ngb::Renderer &r) { r.set_body_poses(poses, memory); });
}

int ngb_bind_geoms(ngb_renderer *h, int32_t gpw, const int32_t *goi, const float *sc) {
    return guarded(h, [&](ngb::Renderer &r) { r.bind_geoms(gpw, goi, sc); });
}

int ngb_set_geom_poses(ngb_renderer *h, const float *xpos, const float *xmat, int32_t memory) {
    return guarded(h, [&](ngb::Renderer &r) { r.set_geom_poses(xpos, xmat, memory); });
}

int ngb_update_mesh(ngb_renderer *h, int32_t mesh, const float *vertices, const float *normals, int32_t memory) {
    return guarded(h, [&](ngb::Renderer &r) { r.update_mesh(mesh, vertices, normals, memory); });
}

int ngb_inspect_mesh(ngb_renderer *h, int32_t mesh, int32_t *node_count, int32_t *triangle_count, int32_t *nodes,
    float *triangles, float *bounds, int32_t *triangle_index) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(mesh >= 0 && mesh < static_cast<int>(r.mesh_tris.size()), "mesh " + std::to_string(mesh) +
            " does not exist: there are " + std::to_string(r.mesh_tris.size()) + " meshes");
        ngb::require(node_count != nullptr && triangle_count != nullptr, "node_count and triangle_count must not be null");
        const int N = r.mesh_nodes[mesh], T = r.mesh_tris[mesh];
        const int node_base = r.mesh_node_base[mesh], tri_base = r.mesh_tri_base[mesh];
        *node_count = N;
        *triangle_count = T;
        if (!nodes && !triangles && !bounds && !triangle_index) return;
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, r.timeout);
        std::vector<int32_t> words(8 * static_cast<size_t>(N));
        CK(cudaMemcpy(words.data(), r.blas.p + 2 * static_cast<size_t>(node_base), words.size() * 4, cudaMemcpyDeviceToHost));
        for (int i = 0; i < N; ++i) words[8 * i + 3] -= words[8 * i + 7] > 0 ? tri_base : node_base;  // mesh-local
        if (nodes) std::memcpy(nodes, words.data(), words.size() * 4);
        if (bounds) {
            std::memcpy(bounds, words.data(), 3 * sizeof(float));
            std::memcpy(bounds + 3, words.data() + 4, 3 * sizeof(float));
        }
        if (triangles)
            CK(cudaMemcpy(triangles, r.tris.p + 3 * static_cast<size_t>(tri_base), 48 * static_cast<size_t>(T),
                cudaMemcpyDeviceToHost));
        if (triangle_index)
            CK(cudaMemcpy(triangle_index, r.tri_index.p + tri_base, 4 * static_cast<size_t>(T), cudaMemcpyDeviceToHost));
    });
}

int ngb_render(ngb_renderer *h, const float *cams, float fov, int32_t spp, uint32_t outputs, int32_t frame,
    int32_t camera_memory, ngb_batch_frame *out) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.check_render(cams, fov, spp, outputs, frame, camera_memory);
        ngb::require(out != nullptr, "out must not be null");
        const size_t px = r.pixels();
        uint8_t *rgb = (outputs & NGB_OUTPUT_RGB) ? r.out_rgb.ensure(3 * px) : nullptr;
        float *depth = (outputs & NGB_OUTPUT_DEPTH) ? r.out_depth.ensure(px) : nullptr;
        float *normal = (outputs & NGB_OUTPUT_NORMAL) ? r.out_normal.ensure(3 * px) : nullptr;
        int32_t *ids = (outputs & NGB_OUTPUT_OBJECT_ID) ? r.out_id.ensure(px) : nullptr;
        r.render(cams, fov, spp, outputs, frame, camera_memory, rgb, depth, normal, ids);
        *out = ngb_batch_frame{NGB_MEMORY_DEVICE, r.device, r.worlds * r.cpw, r.width, r.rows(), rgb, depth, normal, ids};
    });
}

int ngb_render_into(ngb_renderer *h, const float *cams, float fov, int32_t spp, uint32_t outputs, int32_t frame,
    int32_t camera_memory, uint8_t *rgb, float *depth, float *normal, int32_t *object_id) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.check_render(cams, fov, spp, outputs, frame, camera_memory);
        ngb::require(!(outputs & NGB_OUTPUT_RGB) || rgb, "rgb must not be null when the picture is asked for");
        ngb::require(!(outputs & NGB_OUTPUT_DEPTH) || depth, "depth must not be null when depth is asked for");
        ngb::require(!(outputs & NGB_OUTPUT_NORMAL) || normal, "normal must not be null when normals are asked for");
        ngb::require(!(outputs & NGB_OUTPUT_OBJECT_ID) || object_id, "object_id must not be null when IDs are asked for");
        r.render(cams, fov, spp, outputs, frame, camera_memory, rgb, depth, normal, object_id);
    });
}

int ngb_render_host(ngb_renderer *h, const float *cams, float fov, int32_t spp, uint32_t outputs, int32_t frame,
    uint8_t *rgb, float *depth, float *normal, int32_t *object_id) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.check_render(cams, fov, spp, outputs, frame, NGB_MEMORY_HOST);
        const size_t px = r.pixels();
        uint8_t *drgb = (outputs & NGB_OUTPUT_RGB) ? r.out_rgb.ensure(3 * px) : nullptr;
        float *ddepth = (outputs & NGB_OUTPUT_DEPTH) ? r.out_depth.ensure(px) : nullptr;
        float *dnormal = (outputs & NGB_OUTPUT_NORMAL) ? r.out_normal.ensure(3 * px) : nullptr;
        int32_t *dids = (outputs & NGB_OUTPUT_OBJECT_ID) ? r.out_id.ensure(px) : nullptr;
        r.render(cams, fov, spp, outputs, frame, NGB_MEMORY_HOST, drgb, ddepth, dnormal, dids);
        if (drgb && rgb) CK(cudaMemcpyAsync(rgb, drgb, 3 * px, cudaMemcpyDeviceToHost, r.stream));
        if (ddepth && depth) CK(cudaMemcpyAsync(depth, ddepth, px * sizeof(float), cudaMemcpyDeviceToHost, r.stream));
        if (dnormal && normal) CK(cudaMemcpyAsync(normal, dnormal, 3 * px * sizeof(float), cudaMemcpyDeviceToHost, r.stream));
        if (dids && object_id) CK(cudaMemcpyAsync(object_id, dids, px * sizeof(int32_t), cudaMemcpyDeviceToHost, r.stream));
        r.queue_error_read();
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, r.timeout);
        if (*r.host_error) throw ngb::CudaFailure(-1, ngb::device_error_message(*r.host_error));
    });
}

int ngb_make_camera(ngb_vec3 position, ngb_vec3 target, ngb_vec3 world_up, float fov, int32_t width, int32_t height,
    ngb_camera *out) {
    if (!out || width <= 0 || height <= 0) {
        ngb::set_global_error("out must not be null and width and height must be positive");
        return NGB_INVALID_ARGUMENT;
    }
    // In double, then rounded (src/renderer.cpp:39-59).
    struct V {
        double x, y, z;
    };
    auto sub = [](V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; };
    auto cross = [](V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
    auto unit = [](V a) {
        const double n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        return V{a.x / n, a.y / n, a.z / n};
    };
    auto f32 = [](V a) { return ngb_vec3{static_cast<float>(a.x), static_cast<float>(a.y), static_cast<float>(a.z)}; };
    const V fwd = unit(sub(V{target.x, target.y, target.z}, V{position.x, position.y, position.z}));
    const V right = unit(cross(fwd, V{world_up.x, world_up.y, world_up.z}));
    const V up = cross(right, fwd);
    *out = ngb_camera{position, f32(right), f32(up), f32(fwd), std::tan(fov * 0.5f),
        static_cast<float>(width) / static_cast<float>(height)};
    ngb::set_global_error("");
    return NGB_OK;
}

int ngb_render_view(ngb_renderer *h, const ngb_camera *camera, int32_t frame, int32_t spp, uint32_t *argb) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.check_view(camera, frame, spp);
        ngb::require(argb != nullptr, "argb must not be null");
        const size_t px = r.pixels();
        r.render(nullptr, 0.0f, spp, NGB_OUTPUT_RGB, frame, NGB_MEMORY_DEVICE, r.out_rgb.ensure(3 * px), nullptr,
            nullptr, nullptr, camera);
        CK(cudaMemcpyAsync(argb, r.view_argb.p, px * sizeof(uint32_t), cudaMemcpyDeviceToHost, r.stream));
        r.queue_error_read();
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, r.timeout);
        if (*r.host_error) throw ngb::CudaFailure(-1, ngb::device_error_message(*r.host_error));
    });
}

int ngb_render_view_frame(ngb_renderer *h, const ngb_camera *camera, int32_t frame, int32_t spp, uint32_t outputs,
    ngb_batch_frame *out) {
    return guarded(h, [&](ngb::Renderer &r) {
        constexpr unsigned ALL = NGB_OUTPUT_RGB | NGB_OUTPUT_DEPTH | NGB_OUTPUT_NORMAL | NGB_OUTPUT_OBJECT_ID;
        r.check_view(camera, frame, spp);
        ngb::require(outputs != 0, "render_frame needs at least one output");
        ngb::require((outputs & ~ALL) == 0, "unknown output bits in " + std::to_string(outputs));
        ngb::require(out != nullptr, "out must not be null");
        const size_t px = r.pixels();
        uint8_t *rgb = (outputs & NGB_OUTPUT_RGB) ? r.out_rgb.ensure(3 * px) : nullptr;
        float *depth = (outputs & NGB_OUTPUT_DEPTH) ? r.out_depth.ensure(px) : nullptr;
        float *normal = (outputs & NGB_OUTPUT_NORMAL) ? r.out_normal.ensure(3 * px) : nullptr;
        int32_t *ids = (outputs & NGB_OUTPUT_OBJECT_ID) ? r.out_id.ensure(px) : nullptr;
        r.render(nullptr, 0.0f, spp, outputs, frame, NGB_MEMORY_DEVICE, rgb, depth, normal, ids, camera);
        *out = ngb_batch_frame{NGB_MEMORY_DEVICE, r.device, 1, r.width, r.rows(), rgb, depth, normal, ids};
    });
}

int ngb_view_pixels(ngb_renderer *h, const uint32_t **argb) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(argb != nullptr, "argb must not be null");
        *argb = r.view_argb.p;
    });
}

int ngb_cast_rays(ngb_renderer *h, const float *o, const float *d, int32_t rays_per_world, float max_distance,
    int32_t memory, ngb_ray_hits *out) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(out != nullptr, "out must not be null");
        r.cast_rays(o, d, rays_per_world, max_distance, memory, out, nullptr, nullptr, nullptr);
    });
}

int ngb_cast_rays_into(ngb_renderer *h, const float *o, const float *d, int32_t rays_per_world, float max_distance,
    int32_t memory, float *distance, float *normal, int32_t *object_id) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(distance != nullptr && normal != nullptr && object_id != nullptr,
            "distance, normal and object_id must not be null");
        ngb_ray_hits out{};
        r.cast_rays(o, d, rays_per_world, max_distance, memory, &out, distance, normal, object_id);
    });
}

int ngb_copy_to_host(ngb_renderer *h, const void *src, void *dst, size_t bytes) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(bytes == 0 || (src != nullptr && dst != nullptr), "src and dst must not be null");
        if (bytes == 0) return;
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, r.stream));
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, r.timeout);
    });
}

int ngb_set_ambient(ngb_renderer *h, float ambient) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(ngb::finite(ambient) && ambient >= 0.0f, "ambient must be 0 or more, got " + ngb::fstr(ambient));
        r.params.ambient = ambient;
    });
}

float ngb_ambient(const ngb_renderer *h) { return h ? h->r.params.ambient : 0.0f; }

int ngb_set_lights(ngb_renderer *h, const ngb_light *lights, int32_t count) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(count >= 0, "counts must not be negative");
        ngb::require(count == 0 || lights != nullptr, "lights must not be null");
        ngb::check_lights(lights, count);
        r.put_lights(lights, count);
    });
}

int ngb_set_environment(ngb_renderer *h, const ngb_environment *e) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(e != nullptr, "environment must not be null");
        ngb::check_environment(*e);
        // The gradient's up axis, normalised in double (src/environment.cpp:31-38).
        const double u[3] = {e->up.x, e->up.y, e->up.z};
        const double un = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        r.params.env_up = make_float3(static_cast<float>(u[0] / un), static_cast<float>(u[1] / un), static_cast<float>(u[2] / un));
        r.params.env_color_up = make_float3(e->color_up.x, e->color_up.y, e->color_up.z);
        r.params.env_color_down = make_float3(e->color_down.x, e->color_down.y, e->color_down.z);
        r.params.env_intensity = e->intensity;
    });
}

int ngb_set_stream(ngb_renderer *h, void *stream) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.stream = stream ? static_cast<cudaStream_t>(stream) : r.own_stream;
    });
}

int ngb_set_sync(ngb_renderer *h, int32_t synchronous, double timeout_seconds) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(timeout_seconds > 0.0, "timeout_seconds must be positive");
        r.synchronous = synchronous != 0;
        r.timeout = timeout_seconds;
    });
}

int ngb_synchronize(ngb_renderer *h, double timeout_seconds) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.queue_error_read();
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, timeout_seconds > 0.0 ? timeout_seconds : r.timeout);
        r.read_timing();
        if (*r.host_error) throw ngb::CudaFailure(-1, ngb::device_error_message(*r.host_error));
    });
}

int32_t ngb_width(const ngb_renderer *h) { return h ? h->r.width : 0; }
int32_t ngb_height(const ngb_renderer *h) { return h ? h->r.height : 0; }
int32_t ngb_world_count(const ngb_renderer *h) { return h ? h->r.worlds : 0; }
int32_t ngb_cameras_per_world(const ngb_renderer *h) { return h ? h->r.cpw : 0; }
int32_t ngb_view_count(const ngb_renderer *h) { return h ? h->r.worlds * h->r.cpw : 0; }
int32_t ngb_instances_per_world(const ngb_renderer *h) { return h ? h->r.per_world : 0; }

float ngb_last_kernel_ms(const ngb_renderer *ch) {
    ngb_renderer *h = const_cast<ngb_renderer *>(ch);
    if (!h) return 0.0f;
    float ms = 0.0f;
    guarded(h, [&](ngb::Renderer &r) {
        if (r.timing_pending) r.wait(r.ev_stop, r.timeout);
        r.read_timing();
        ms = r.kernel_ms;
    });
    return ms;
}

int ngb_last_stage_ms(ngb_renderer *h, float *ms, int32_t capacity, int32_t *count) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(ms != nullptr && count != nullptr && capacity >= 0, "ms and count must not be null");
        if (r.timing_pending) r.wait(r.ev_stop, r.timeout);
        r.read_timing();
        *count = r.stages;
        for (int i = 0; i < r.stages && i < capacity; ++i) ms[i] = r.stage_ms[i];
    });
}

int ngb_build_meshes(const ngb_mesh *meshes, int32_t mesh_count, int32_t *node_count, int32_t *triangle_count,
    int32_t *nodes, float *triangles, int32_t *roots, float *bounds, int32_t *triangle_index) {
    try {
        ngb::require(mesh_count >= 0 && (mesh_count == 0 || meshes) && node_count && triangle_count,
            "meshes, node_count and triangle_count must not be null");
        ngb_scene s{};
        s.meshes = meshes;
        s.mesh_count = mesh_count;
        ngb::check_meshes(s);
        const ngb::BuiltMeshes b = ngb::build_meshes(s);
        *node_count = static_cast<int32_t>(b.nodes.size() / 8);
        *triangle_count = static_cast<int32_t>(b.triangle_index.size());
        if (nodes) std::memcpy(nodes, b.nodes.data(), b.nodes.size() * sizeof(float));
        if (triangles) std::memcpy(triangles, b.triangles.data(), b.triangles.size() * sizeof(float));
        if (roots) std::memcpy(roots, b.roots.data(), b.roots.size() * sizeof(int32_t));
        if (bounds) std::memcpy(bounds, b.bounds.data(), b.bounds.size() * sizeof(float));
        if (triangle_index) std::memcpy(triangle_index, b.triangle_index.data(), b.triangle_index.size() * sizeof(int32_t));
        g_create_error.clear();
        return NGB_OK;
    } catch (const ngb::InvalidArgument &e) {
        g_create_error = e.what();
        return NGB_INVALID_ARGUMENT;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return NGB_CUDA_ERROR;
    }
}

int ngb_set_tuning(ngb_renderer *h, int32_t kernel, int32_t threads_per_block, int32_t refill_lanes,
    int32_t registers, int32_t leaf_batch) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(kernel >= 0 && kernel <= 3,
            "kernel must be 0 (automatic), 1 (per pixel), 2 (persistent) or 3 (tiles)");
        if (kernel == 3) {
            const bool built = (threads_per_block == 128 && (registers == 48 || registers == 56 || registers == 64 ||
                registers == 80)) || (threads_per_block == 256 && registers == 64);
            ngb::require(built, "for the tile kernel, threads_per_block and registers must be one of 128/48, 128/56, "
                "128/64, 128/80, 256/64");
            r.kernel_choice = kernel;
            r.tile_tuning.threads = threads_per_block;
            r.tile_tuning.registers = registers;
            return;
        }
        const bool built = (threads_per_block == 128 && (registers == 48 || registers == 64 || registers == 72)) ||
            (threads_per_block == 256 && (registers == 48 || registers == 64)) || (threads_per_block == 64 && registers == 64);
        ngb::require(built, "threads_per_block and registers must be one of 128/48, 128/64, 128/72, 256/48, 256/64, 64/64");
        ngb::require(refill_lanes >= 1 && refill_lanes <= 32, "refill_lanes must be 1 to 32");
        ngb::require(leaf_batch >= 1 && leaf_batch <= 32, "leaf_batch must be 1 to 32");
        r.kernel_choice = kernel;
        r.tuning = ngb::PersistentTuning{threads_per_block, refill_lanes, registers, leaf_batch};
    });
}

int ngb_set_tile_shape(ngb_renderer *h, int32_t tiles_per_fetch, int32_t paired) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(tiles_per_fetch >= 1 && tiles_per_fetch <= 8, "tiles_per_fetch must be 1 to 8, got " +
            std::to_string(tiles_per_fetch));
        ngb::require(paired == 0 || paired == 1, "paired must be 0 or 1");
        r.tile_tuning.tile_fetch = tiles_per_fetch;
        r.tile_tuning.tile_pairs = paired;
    });
}

int ngb_set_ray_kernel(ngb_renderer *h, int32_t kernel) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(kernel >= 0 && kernel <= 3,
            "kernel must be 0 (automatic), 1 (per thread), 2 (persistent) or 3 (warp packets)");
        r.ray_kernel = kernel;
    });
}

int ngb_set_build(ngb_renderer *h, int32_t mode) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(mode >= 0 && mode <= 2, "mode must be 0 (automatic), 1 (per world) or 2 (global)");
        ngb::require(mode != 1 || r.per_world <= ngb::MAX_PER_WORLD,
            "the per-world build takes at most " + std::to_string(ngb::MAX_PER_WORLD) + " instances per world");
        r.build_mode = mode;
    });
}

int ngb_inject_allocation_failure(int32_t after) {
    ngb::g_fail_allocation = after < 0 ? -1 : after;
    return NGB_OK;
}

int64_t ngb_device_bytes(void) { return ngb::g_device_bytes.load(); }

int ngb_set_rows(ngb_renderer *h, int32_t first, int32_t count) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(!r.uneven, "worlds of uneven sizes render whole images");
        ngb::require(first >= 0 && count >= 1 && static_cast<long long>(first) + count <= r.height,
            "rows [" + std::to_string(first) + ", " + std::to_string(static_cast<long long>(first) + count) +
            ") are not a non-empty range of the image's " + std::to_string(r.height) + " rows");
        r.band_first = first;
        r.band_rows = count == r.height ? 0 : count;
    });
}

int ngb_rows(const ngb_renderer *h, int32_t *first, int32_t *count) {
    if (!h || !first || !count) return NGB_INVALID_ARGUMENT;
    *first = h->r.band_first;
    *count = h->r.rows();
    return NGB_OK;
}

int ngb_srgb_thresholds(float *thresholds) {
    if (!thresholds) return NGB_INVALID_ARGUMENT;
    ngb::srgb_thresholds(thresholds);
    return NGB_OK;
}

int ngb_record_hits(ngb_renderer *h, int32_t on) {
    return guarded(h, [&](ngb::Renderer &r) {
        r.record_hits = on != 0;
        r.ext_instance = r.ext_triangle = nullptr;
        r.ext_u = r.ext_v = nullptr;
    });
}

int ngb_record_hits_into(ngb_renderer *h, int32_t *instance, int32_t *triangle, float *u, float *v) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(instance && triangle && u && v, "instance, triangle, u and v must all be given");
        r.record_hits = true;
        r.ext_instance = instance;
        r.ext_triangle = triangle;
        r.ext_u = u;
        r.ext_v = v;
    });
}

int ngb_inspect_tlas(ngb_renderer *h, uint64_t *keys, int32_t *sorted_ids, int32_t *nodes, int32_t *roots,
    float *matrices) {
    return guarded(h, [&](ngb::Renderer &r) {
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, r.timeout);
        const size_t n = static_cast<size_t>(r.n);
        if (n == 0) return;
        if (keys) CK(cudaMemcpy(keys, r.keys.p, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        if (sorted_ids) CK(cudaMemcpy(sorted_ids, r.sorted_ids.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (nodes) CK(cudaMemcpy(nodes, r.tlas.p, (2 * n - 1) * 32, cudaMemcpyDeviceToHost));
        if (roots) CK(cudaMemcpy(roots, r.roots.p, r.worlds * sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (matrices) CK(cudaMemcpy(matrices, r.matrices.p, n * 48, cudaMemcpyDeviceToHost));
    });
}

int ngb_copy_hits(ngb_renderer *h, int32_t *instance, int32_t *triangle, float *u, float *v) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(r.hits_instance() != nullptr, "no hit records: call ngb_record_hits(r, 1) before rendering");
        const size_t px = r.pixels() * 4;
        if (instance) CK(cudaMemcpyAsync(instance, r.hits_instance(), px, cudaMemcpyDeviceToDevice, r.stream));
        if (triangle) CK(cudaMemcpyAsync(triangle, r.hits_triangle(), px, cudaMemcpyDeviceToDevice, r.stream));
        if (u) CK(cudaMemcpyAsync(u, r.hits_u(), px, cudaMemcpyDeviceToDevice, r.stream));
        if (v) CK(cudaMemcpyAsync(v, r.hits_v(), px, cudaMemcpyDeviceToDevice, r.stream));
        r.finish();
    });
}

int ngb_depth_normal_adjoint(ngb_renderer *h, const float *matrices, const float *cameras, float fov,
    const int32_t *hit_instance, const int32_t *hit_triangle, const float *hit_u, const float *hit_v, const float *depth,
    const float *grad_depth, const float *grad_normal, float *grad_matrices, float *grad_cameras) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(matrices && cameras && hit_instance && hit_triangle && hit_u && hit_v && depth && grad_depth &&
            grad_matrices && grad_cameras, "only grad_normal may be null");
        ngb::require(fov > 0.0f && fov < 3.14159265f, "fov must be between 0 and pi radians");
        ngb::require(!r.uneven, "the adjoint takes worlds of one size");
        ngb::AdjointArgs a{};
        a.matrices = matrices;
        a.cameras = cameras;
        a.fov_scale = std::tan(fov * 0.5f);
        a.aspect = static_cast<float>(r.width) / static_cast<float>(r.height);
        a.width = r.width;
        a.height = r.height;
        a.row_first = r.band_first;
        a.rows = r.rows();
        a.cameras_per_world = r.cpw;
        a.views = r.worlds * r.cpw;
        a.hit_instance = hit_instance;
        a.hit_triangle = hit_triangle;
        a.hit_u = hit_u;
        a.hit_v = hit_v;
        a.depth = depth;
        a.grad_depth = grad_depth;
        a.grad_normal = grad_normal;
        a.grad_matrices = grad_matrices;
        a.grad_cameras = grad_cameras;
        a.tri_of_local = r.tri_of_local.p;
        a.slot_tri_base = r.slot_tri_base.p;
        ngb::Range range("ngb depth_normal_adjoint");
        CK(cudaEventRecord(r.ev_start, r.stream));
        CK(ngb::launch_depth_normal_adjoint(r.params, a, r.stream));
        CK(cudaEventRecord(r.ev_stop, r.stream));
        r.stages = 1;
        r.timing_pending = true;
        r.finish();
    });
}

int ngb_inspect_hits(ngb_renderer *h, int32_t *instance, int32_t *triangle, float *u, float *v) {
    return guarded(h, [&](ngb::Renderer &r) {
        ngb::require(r.hits_instance() != nullptr, "no hit records: call ngb_record_hits(r, 1) before rendering");
        CK(cudaEventRecord(r.ev_done, r.stream));
        r.wait(r.ev_done, r.timeout);
        const size_t px = r.pixels();
        if (instance) CK(cudaMemcpy(instance, r.hits_instance(), px * 4, cudaMemcpyDeviceToHost));
        if (triangle) CK(cudaMemcpy(triangle, r.hits_triangle(), px * 4, cudaMemcpyDeviceToHost));
        if (u) CK(cudaMemcpy(u, r.hits_u(), px * 4, cudaMemcpyDeviceToHost));
        if (v) CK(cudaMemcpy(v, r.hits_v(), px * 4, cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"
