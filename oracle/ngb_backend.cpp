// Test infrastructure: the reference-side binding a maintainer would add so that the REFERENCE's own
// BatchRenderer and Renderer (neraulgraphics 0.5.0, src/batch.cpp, src/renderer.cpp, compiled from its sources by
// oracle/Makefile) draw through this library. It implements the reference's backend seam, detail::Backend
// (src/backend.h:36-85), on the C ABI of include/ngb.h, and provides detail::make_cuda_backend (src/backend.h:88)
// in place of the reference's CUDA backend, so Device::Cuda picks it. Linked into oracle/_ref/libngref_ngb.so
// with the reference's library files and ref_harness.cpp; nothing in the product links this file.
//
// The seam hands a backend the meshes' built trees (SceneInput::built) but not the meshes, and ngb_create builds
// its trees from the meshes themselves (node for node the reference's build). The meshes the caller gave reach
// this binding through ngref_use_meshes, called just before the renderer is made: the stand-in for the one line
// a maintainer would add to SceneInput, a reference to the meshes.

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <neraulgraphics/batch.h>
#include <neraulgraphics/renderer.h>

#include "backend.h"

#include "../include/ngb.h"

using namespace neraulgraphics;

namespace {

thread_local const ngb_mesh *g_meshes = nullptr;
thread_local int g_mesh_count = 0;

ngb_vec3 v3(const Vec3 &v) { return ngb_vec3{v.x, v.y, v.z}; }

ngb_material material(const Material &m) {
    return ngb_material{v3(m.diffuse_color), m.diffuse_albedo, m.specular_albedo, m.reflectivity, m.specular_exponent,
        m.roughness, m.metallic, v3(m.emission), m.transmission, m.ior};
}

ngb_light light(const Light &l) {
    return ngb_light{v3(l.position), l.intensity, l.radius, l.falloff, v3(l.direction), l.spot_angle, l.spot_softness,
        v3(l.color)};
}

[[noreturn]] void raise(ngb_renderer *h, int status) {
    const std::string message = ngb_last_error(h);
    if (status == NGB_INVALID_ARGUMENT) throw std::invalid_argument(message);
    if (status == NGB_LOGIC_ERROR) throw std::logic_error(message);
    throw CudaError(-1, message);
}

class NgbBackend final : public detail::Backend {
public:
    explicit NgbBackend(const detail::SceneInput &s) : width_(s.width), height_(s.height) {
        if (!s.textures.empty()) throw std::invalid_argument("textures are not supported by this backend");
        if (!s.instances.empty() && !g_meshes) throw std::logic_error("ngref_use_meshes was not called before the renderer");
        std::vector<ngb_sphere> spheres;
        for (const Sphere &sp : s.spheres) spheres.push_back(ngb_sphere{v3(sp.center), sp.radius, material(sp.material)});
        std::vector<ngb_light> lights;
        for (const Light &l : s.lights) lights.push_back(light(l));
        std::vector<ngb_instance> instances;
        for (const Instance &in : s.instances) {
            if (in.texture >= 0 || in.normal_texture >= 0 || in.orm_texture >= 0)
                throw std::invalid_argument("textures are not supported by this backend");
            ngb_instance out{in.mesh, {}, material(in.material)};
            std::memcpy(out.transform, in.transform.m, sizeof(out.transform));
            instances.push_back(out);
        }
        ngb_scene scene{};
        scene.width = s.width;
        scene.height = s.height;
        scene.world_count = s.worlds;
        scene.cameras_per_world = s.cameras_per_world;
        scene.spheres = spheres.data();
        scene.sphere_count = static_cast<int32_t>(spheres.size());
        scene.lights = lights.data();
        scene.light_count = static_cast<int32_t>(lights.size());
        scene.floor = ngb_plane{s.floor.y, s.floor.half_extent_x, s.floor.z_min, s.floor.z_max, s.floor.checker_scale,
            material(s.floor.material)};
        scene.meshes = s.instances.empty() ? nullptr : g_meshes;
        scene.mesh_count = s.instances.empty() ? 0 : g_mesh_count;
        scene.instances = instances.data();
        scene.instance_count = static_cast<int32_t>(instances.size());
        scene.device = 0;
        const int status = ngb_create(&scene, &h_);
        if (status != NGB_OK) raise(nullptr, status);
        instance_count_ = static_cast<int>(instances.size());
    }
    ~NgbBackend() override { ngb_destroy(h_); }

    const uint32_t *render(const Camera &camera, int frame, int samples_per_frame) override {
        const ngb_camera cam = view(camera);
        pixels_.resize(static_cast<size_t>(width_) * height_);
        check(ngb_render_view(h_, &cam, frame, samples_per_frame, pixels_.data()));
        return pixels_.data();
    }

    Frame render_frame(const Camera &camera, int frame, int samples_per_frame, unsigned outputs) override {
        const ngb_camera cam = view(camera);
        ngb_batch_frame f;
        check(ngb_render_view_frame(h_, &cam, frame, samples_per_frame, outputs, &f));
        check(ngb_synchronize(h_, 120.0));
        return Frame{Memory::Device, f.device_id, f.width, f.height, f.rgb, f.depth, f.normal, f.object_id};
    }

    RayHits cast_rays(const float *origins, const float *directions, int count, float max_distance,
        Memory memory) override {
        ngb_ray_hits hits;
        check(ngb_cast_rays(h_, origins, directions, count, max_distance, memory == Memory::Device, &hits));
        check(ngb_synchronize(h_, 120.0));
        return RayHits{Memory::Device, hits.device_id, hits.count, hits.distance, hits.normal, hits.object_id};
    }

    void copy_to_host(const void *src, void *dst, size_t bytes) const override {
        check(ngb_copy_to_host(h_, src, dst, bytes));
    }

    void set_instance_transforms(const std::vector<Transform> &transforms) override {
        std::vector<float> m(12 * transforms.size());
        for (size_t i = 0; i < transforms.size(); ++i) std::memcpy(&m[12 * i], transforms[i].m, 12 * sizeof(float));
        check(ngb_set_instance_transforms(h_, m.data(), NGB_MEMORY_HOST));
    }

    void set_instance_matrices(const float *matrices, Memory memory) override {
        check(ngb_set_instance_transforms(h_, matrices, memory == Memory::Device));
    }

    void bind_bodies(const BodyBinding &b) override {
        check(ngb_bind_bodies(h_, b.bodies_per_world, b.body_of_instance.data(), b.local_pose.data(), b.scale.data()));
    }

    void set_body_poses(const float *poses, Memory memory) override {
        check(ngb_set_body_poses(h_, poses, memory == Memory::Device));
    }

    BatchFrame render_batch(const float *cameras, Memory memory, float fov, int spp, unsigned outputs,
        int frame) override {
        ngb_batch_frame f;
        check(ngb_render(h_, cameras, fov, spp, outputs, frame, memory == Memory::Device, &f));
        check(ngb_synchronize(h_, 120.0));
        return BatchFrame{Memory::Device, f.device_id, f.views, f.width, f.height, f.rgb, f.depth, f.normal, f.object_id};
    }

    RayHits cast_rays_batch(const float *origins, const float *directions, int rays_per_world, float max_distance,
        Memory memory) override {
        return cast_rays(origins, directions, rays_per_world, max_distance, memory);
    }

    void set_lights(const std::vector<Light> &lights) override {
        std::vector<ngb_light> out;
        for (const Light &l : lights) out.push_back(light(l));
        check(ngb_set_lights(h_, out.data(), static_cast<int32_t>(out.size())));
    }

    void set_ambient(float ambient) override { check(ngb_set_ambient(h_, ambient)); }
    float ambient() const override { return ngb_ambient(h_); }

    void set_render_mode(RenderMode mode, const PathTracing &) override {
        if (mode != RenderMode::Classic) throw std::invalid_argument("this backend draws the classic picture only");
    }
    RenderMode render_mode() const override { return RenderMode::Classic; }

    void set_environment(const Environment &e) override {
        if (!e.map.empty()) throw std::invalid_argument("this backend draws the gradient sky only");
        const ngb_environment env{v3(e.up), v3(e.color_up), v3(e.color_down), e.intensity};
        check(ngb_set_environment(h_, &env));
    }

    float last_kernel_ms() const override { return ngb_last_kernel_ms(h_); }
    Device device() const override { return Device::Cuda; }

private:
    ngb_renderer *h_ = nullptr;
    int width_, height_, instance_count_ = 0;
    std::vector<uint32_t> pixels_;

    void check(int status) const {
        if (status != NGB_OK) raise(h_, status);
    }

    static ngb_camera view(const Camera &c) {
        return ngb_camera{v3(c.position), v3(c.right), v3(c.up), v3(c.forward), c.fov_scale, c.aspect};
    }
};

}  // namespace

namespace neraulgraphics::detail {

// The reference's CUDA backend, replaced (src/backend.h:88): Device::Cuda now draws through this library.
std::unique_ptr<Backend> make_cuda_backend(const SceneInput &scene) { return std::make_unique<NgbBackend>(scene); }

bool cuda_usable() { return true; }

}  // namespace neraulgraphics::detail

extern "C" void ngref_use_meshes(const ngb_mesh *meshes, int count) {
    g_meshes = meshes;
    g_mesh_count = count;
}
