// Test infrastructure: a C ABI over the REFERENCE implementation (neraulgraphics 0.5.0, compiled from its
// own sources by oracle/Makefile into oracle/_ref/), so the Python tests and bench.py's reference arm can
// drive it through ctypes. Nothing in the product links this file.
//
// It exposes:
//   - BatchRenderer on Device::Cpu (or Device::Cuda when the library was built with the reference's CUDA
//     backend) with the scene passed as the same plain structs the product's ABI takes (include/ngb.h);
//   - its single-view Renderer (render's running average, render_frame) on the same structs;
//   - the reference's host helpers the product restates, for bit-exact pinning: detail::build_meshes
//     (src/mesh_build.cpp:91-157), detail::body_poses_to_matrices (src/instances.cpp:137-164),
//     make_icosphere / make_box / make_transform (src/mesh.cpp), make_camera (src/renderer.cpp:39-59),
//     detail::invert_affine and detail::transform_aabb (src/mesh_build.cpp:159-197).

#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <neraulgraphics/batch.h>
#include <neraulgraphics/mesh.h>
#include <neraulgraphics/renderer.h>

#include "instances.h"
#include "mesh_build.h"

#include "../include/ngb.h"

using namespace neraulgraphics;

namespace {

thread_local std::string g_error;

int fail(const std::exception &e) {
    g_error = e.what();
    if (dynamic_cast<const std::invalid_argument *>(&e)) return NGB_INVALID_ARGUMENT;
    if (dynamic_cast<const CudaError *>(&e)) return NGB_CUDA_ERROR;
    if (dynamic_cast<const std::logic_error *>(&e)) return NGB_LOGIC_ERROR;
    return NGB_CUDA_ERROR;
}

Vec3 v3(const ngb_vec3 &v) { return Vec3{v.x, v.y, v.z}; }

Material mat(const ngb_material &m) {
    Material out{v3(m.diffuse_color), m.diffuse_albedo, m.specular_albedo, m.reflectivity, m.specular_exponent};
    out.roughness = m.roughness;
    out.metallic = m.metallic;
    out.emission = v3(m.emission);
    out.transmission = m.transmission;
    out.ior = m.ior;
    return out;
}

struct Scene {
    std::vector<Sphere> spheres;
    std::vector<Light> lights;
    Plane floor{};
    std::vector<Mesh> meshes;
    std::vector<Instance> instances;
};

Scene convert(const ngb_scene &s) {
    Scene out;
    for (int i = 0; i < s.sphere_count; ++i)
        out.spheres.push_back(Sphere{v3(s.spheres[i].center), s.spheres[i].radius, mat(s.spheres[i].material)});
    for (int i = 0; i < s.light_count; ++i) {
        const ngb_light &l = s.lights[i];
        Light L{v3(l.position), l.intensity, l.radius};
        L.falloff = l.falloff;
        L.direction = v3(l.direction);
        L.spot_angle = l.spot_angle;
        L.spot_softness = l.spot_softness;
        L.color = v3(l.color);
        out.lights.push_back(L);
    }
    out.floor = Plane{s.floor.y, s.floor.half_extent_x, s.floor.z_min, s.floor.z_max, s.floor.checker_scale,
        mat(s.floor.material)};
    for (int m = 0; m < s.mesh_count; ++m) {
        const ngb_mesh &src = s.meshes[m];
        Mesh mesh;
        for (int v = 0; v < src.vertex_count; ++v)
            mesh.vertices.push_back(Vec3{src.vertices[3 * v], src.vertices[3 * v + 1], src.vertices[3 * v + 2]});
        mesh.indices.assign(src.indices, src.indices + src.index_count);
        if (src.normals)
            for (int v = 0; v < src.vertex_count; ++v)
                mesh.normals.push_back(Vec3{src.normals[3 * v], src.normals[3 * v + 1], src.normals[3 * v + 2]});
        out.meshes.push_back(std::move(mesh));
    }
    for (int i = 0; i < s.instance_count; ++i) {
        Instance inst{};
        inst.mesh = s.instances[i].mesh;
        std::memcpy(inst.transform.m, s.instances[i].transform, sizeof(inst.transform.m));
        inst.material = mat(s.instances[i].material);
        out.instances.push_back(inst);
    }
    return out;
}

struct Handle {
    std::unique_ptr<BatchRenderer> batch;
};

struct ViewHandle {
    std::unique_ptr<Renderer> view;
};

Camera camera_of(const ngb_camera &c) {
    return Camera{v3(c.position), v3(c.right), v3(c.up), v3(c.forward), c.fov_scale, c.aspect};
}

}  // namespace

extern "C" {

const char *ngref_last_error(void) { return g_error.c_str(); }

// Sets NERAULGRAPHICS_THREADS, which the CPU backend reads at every parallel loop (src/cpu_backend.cpp:94-101).
void ngref_set_threads(int threads) {
    const std::string v = std::to_string(threads);
    setenv("NERAULGRAPHICS_THREADS", v.c_str(), 1);
}

// device: 0 for Device::Cpu, 1 for Device::Cuda (only in a library built with the reference's CUDA backend).
int ngref_create(const ngb_scene *scene, int device, void **out) {
    *out = nullptr;
    try {
        const Scene s = convert(*scene);
        auto h = std::make_unique<Handle>();
        h->batch = std::make_unique<BatchRenderer>(scene->width, scene->height, scene->world_count,
            scene->cameras_per_world, s.spheres, s.lights, s.floor, s.meshes, s.instances, std::vector<Texture>{},
            device == 1 ? Device::Cuda : Device::Cpu);
        *out = h.release();
        g_error.clear();
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

void ngref_destroy(void *h) { delete static_cast<Handle *>(h); }

int ngref_set_instance_transforms(void *h, const float *matrices, int memory) {
    try {
        static_cast<Handle *>(h)->batch->set_instance_transforms(matrices, memory ? Memory::Device : Memory::Host);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int ngref_bind_bodies(void *h, int bodies_per_world, const int *body_of_instance, const float *local_pose,
    const float *scale, int instances) {
    try {
        BodyBinding b;
        b.bodies_per_world = bodies_per_world;
        b.body_of_instance.assign(body_of_instance, body_of_instance + instances);
        b.local_pose.assign(local_pose, local_pose + 7 * instances);
        b.scale.assign(scale, scale + 3 * instances);
        static_cast<Handle *>(h)->batch->bind_bodies(b);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int ngref_set_body_poses(void *h, const float *poses, int memory) {
    try {
        static_cast<Handle *>(h)->batch->set_body_poses(poses, memory ? Memory::Device : Memory::Host);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int ngref_set_ambient(void *h, float ambient) {
    try {
        static_cast<Handle *>(h)->batch->set_ambient(ambient);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Renders from host cameras and copies every asked-for image into the caller's host buffers.
int ngref_render_host(void *h, const float *cams, float fov, int spp, unsigned outputs, int frame, uint8_t *rgb,
    float *depth, float *normal, int32_t *ids) {
    try {
        const HostBatchFrame f = static_cast<Handle *>(h)->batch->render_host(cams, fov, spp, outputs, frame);
        if (rgb && !f.rgb.empty()) std::memcpy(rgb, f.rgb.data(), f.rgb.size());
        if (depth && !f.depth.empty()) std::memcpy(depth, f.depth.data(), f.depth.size() * sizeof(float));
        if (normal && !f.normal.empty()) std::memcpy(normal, f.normal.data(), f.normal.size() * sizeof(float));
        if (ids && !f.object_id.empty()) std::memcpy(ids, f.object_id.data(), f.object_id.size() * sizeof(int32_t));
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Renders and leaves the images where the backend keeps them (device memory for Device::Cuda). For timing.
int ngref_render(void *h, const float *cams, float fov, int spp, unsigned outputs, int frame, int camera_memory,
    ngb_batch_frame *out) {
    try {
        const BatchFrame f = static_cast<Handle *>(h)->batch->render(cams, fov, spp, outputs, frame,
            camera_memory ? Memory::Device : Memory::Host);
        if (out) {
            out->memory = f.memory == Memory::Device ? NGB_MEMORY_DEVICE : NGB_MEMORY_HOST;
            out->device_id = f.device_id;
            out->views = f.views;
            out->width = f.width;
            out->height = f.height;
            out->rgb = f.rgb;
            out->depth = f.depth;
            out->normal = f.normal;
            out->object_id = f.object_id;
        }
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int ngref_cast_rays_host(void *h, const float *origins, const float *directions, int rays_per_world, int worlds,
    float max_distance, float *distance, float *normal, int32_t *ids) {
    try {
        const size_t n = static_cast<size_t>(rays_per_world >= 0 ? rays_per_world : 0) * worlds * 3;
        const std::vector<float> o(origins, origins + n), d(directions, directions + n);
        const HostRayHits r = static_cast<Handle *>(h)->batch->cast_rays_host(o, d, rays_per_world, max_distance);
        if (distance) std::memcpy(distance, r.distance.data(), r.distance.size() * sizeof(float));
        if (normal) std::memcpy(normal, r.normal.data(), r.normal.size() * sizeof(float));
        if (ids) std::memcpy(ids, r.object_id.data(), r.object_id.size() * sizeof(int32_t));
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// BatchRenderer::cast_rays with the rays in device memory; the hits stay in the renderer's device buffers.
int ngref_cast_rays_device(void *h, const float *origins, const float *directions, int rays_per_world,
    float max_distance) {
    try {
        static_cast<Handle *>(h)->batch->cast_rays(origins, directions, rays_per_world, max_distance, Memory::Device);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

float ngref_last_kernel_ms(void *h) { return static_cast<Handle *>(h)->batch->last_kernel_ms(); }

int ngref_device(void *h) { return static_cast<Handle *>(h)->batch->device() == Device::Cuda ? 1 : 0; }

// ---- host helpers, for pinning the product's restatements bit-exactly -------------------------------------

// detail::build_meshes. Call once with null outputs to learn the sizes (node, triangle and mesh counts), then
// again with buffers: nodes as 8 words each (bvh::Node, src/bvh.h:30-35), triangles as 12 floats each,
// roots and bounds (6 floats) per mesh.
int ngref_build_meshes(const ngb_mesh *meshes, int mesh_count, int *node_count, int *triangle_count, int32_t *nodes,
    float *triangles, int32_t *roots, float *bounds) {
    try {
        ngb_scene s{};
        s.meshes = meshes;
        s.mesh_count = mesh_count;
        const Scene sc = convert(s);
        const detail::BuiltMeshes b = detail::build_meshes(sc.meshes);
        *node_count = static_cast<int>(b.nodes.size());
        *triangle_count = static_cast<int>(b.triangles.size() / 12);
        if (nodes) std::memcpy(nodes, b.nodes.data(), b.nodes.size() * sizeof(bvh::Node));
        if (triangles) std::memcpy(triangles, b.triangles.data(), b.triangles.size() * sizeof(float));
        if (roots) std::memcpy(roots, b.roots.data(), b.roots.size() * sizeof(int));
        if (bounds)
            for (size_t m = 0; m < b.bounds.size(); ++m) {
                std::memcpy(bounds + 6 * m, b.bounds[m].lo, 3 * sizeof(float));
                std::memcpy(bounds + 6 * m + 3, b.bounds[m].hi, 3 * sizeof(float));
            }
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// detail::body_poses_to_matrices (the host twin, computed in double).
int ngref_body_poses_to_matrices(int bodies_per_world, const int *body_of_instance, const float *local_pose,
    const float *scale, int instances, int worlds, const float *poses, float *out) {
    try {
        BodyBinding b;
        b.bodies_per_world = bodies_per_world;
        b.body_of_instance.assign(body_of_instance, body_of_instance + instances);
        b.local_pose.assign(local_pose, local_pose + 7 * instances);
        b.scale.assign(scale, scale + 3 * instances);
        detail::body_poses_to_matrices(b, worlds, poses, out);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// make_icosphere / make_box: call with null buffers for the counts, then with buffers.
int ngref_make_icosphere(float radius, int subdivisions, int *vertex_count, int *index_count, float *vertices,
    uint32_t *indices) {
    try {
        const Mesh m = make_icosphere(radius, subdivisions);
        *vertex_count = static_cast<int>(m.vertices.size());
        *index_count = static_cast<int>(m.indices.size());
        if (vertices) std::memcpy(vertices, m.vertices.data(), m.vertices.size() * sizeof(Vec3));
        if (indices) std::memcpy(indices, m.indices.data(), m.indices.size() * sizeof(uint32_t));
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int ngref_make_box(float hx, float hy, float hz, float *vertices, uint32_t *indices) {
    const Mesh m = make_box(Vec3{hx, hy, hz});
    std::memcpy(vertices, m.vertices.data(), m.vertices.size() * sizeof(Vec3));
    std::memcpy(indices, m.indices.data(), m.indices.size() * sizeof(uint32_t));
    return NGB_OK;
}

int ngref_make_transform(const float *position, const float *quat, float scale, float *out) {
    try {
        const Transform t = make_transform(Vec3{position[0], position[1], position[2]},
            Quat{quat[0], quat[1], quat[2], quat[3]}, scale);
        std::memcpy(out, t.m, sizeof(t.m));
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// make_camera, returned as the camera-to-world matrix the batch API takes (tests/test_batch.cpp:59-62).
void ngref_camera_matrix(const float *position, const float *target, const float *world_up, float fov, int width,
    int height, float *out) {
    const Camera c = make_camera(Vec3{position[0], position[1], position[2]}, Vec3{target[0], target[1], target[2]},
        Vec3{world_up[0], world_up[1], world_up[2]}, fov, width, height);
    const float m[12] = {c.right.x, c.up.x, -c.forward.x, c.position.x, c.right.y, c.up.y, -c.forward.y,
        c.position.y, c.right.z, c.up.z, -c.forward.z, c.position.z};
    std::memcpy(out, m, sizeof(m));
}

int ngref_invert_affine(const float *m, float *out) {
    Transform t, inv;
    std::memcpy(t.m, m, sizeof(t.m));
    const bool ok = detail::invert_affine(t, inv);
    std::memcpy(out, inv.m, sizeof(inv.m));
    return ok ? 1 : 0;
}

void ngref_transform_aabb(const float *m, const float *box, float *out) {
    Transform t;
    std::memcpy(t.m, m, sizeof(t.m));
    bvh::Aabb b{{box[0], box[1], box[2]}, {box[3], box[4], box[5]}};
    const bvh::Aabb r = detail::transform_aabb(t, b);
    std::memcpy(out, r.lo, 3 * sizeof(float));
    std::memcpy(out + 3, r.hi, 3 * sizeof(float));
}

// The reference's single-view Renderer (include/neraulgraphics/renderer.h:135-277) over the same plain scene
// structs: scene->width and height are its frame; world_count and cameras_per_world are not read.
int ngref_view_create(const ngb_scene *scene, int device, void **out) {
    *out = nullptr;
    try {
        const Scene s = convert(*scene);
        auto h = std::make_unique<ViewHandle>();
        h->view = std::make_unique<Renderer>(scene->width, scene->height, s.spheres, s.lights, s.floor, s.meshes,
            s.instances, std::vector<Texture>{}, device == 1 ? Device::Cuda : Device::Cpu);
        *out = h.release();
        g_error.clear();
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

void ngref_view_destroy(void *h) { delete static_cast<ViewHandle *>(h); }

int ngref_view_set_matrices(void *h, const float *matrices) {
    try {
        static_cast<ViewHandle *>(h)->view->set_instance_matrices(matrices, Memory::Host);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int ngref_view_set_ambient(void *h, float ambient) {
    try {
        static_cast<ViewHandle *>(h)->view->set_ambient(ambient);
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Renderer::render: width x height 0xAARRGGBB pixels into argb.
int ngref_view_render(void *h, const ngb_camera *camera, int frame, int spp, uint32_t *argb) {
    try {
        Renderer &r = *static_cast<ViewHandle *>(h)->view;
        const uint32_t *p = r.render(camera_of(*camera), frame, spp);
        std::memcpy(argb, p, static_cast<size_t>(r.width()) * r.height() * sizeof(uint32_t));
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Renderer::render_frame_host into the caller's buffers (any may be NULL).
int ngref_view_render_frame(void *h, const ngb_camera *camera, int frame, int spp, unsigned outputs, uint8_t *rgb,
    float *depth, float *normal, int32_t *ids) {
    try {
        const HostFrame f = static_cast<ViewHandle *>(h)->view->render_frame_host(camera_of(*camera), frame, spp, outputs);
        if (rgb && !f.rgb.empty()) std::memcpy(rgb, f.rgb.data(), f.rgb.size());
        if (depth && !f.depth.empty()) std::memcpy(depth, f.depth.data(), f.depth.size() * sizeof(float));
        if (normal && !f.normal.empty()) std::memcpy(normal, f.normal.data(), f.normal.size() * sizeof(float));
        if (ids && !f.object_id.empty()) std::memcpy(ids, f.object_id.data(), f.object_id.size() * sizeof(int32_t));
        return NGB_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// make_camera (src/renderer.cpp:39-59), the whole Camera: position, right, up, forward, fov_scale, aspect.
void ngref_make_camera(const float *position, const float *target, const float *world_up, float fov, int width,
    int height, float *out) {
    const Camera c = make_camera(Vec3{position[0], position[1], position[2]}, Vec3{target[0], target[1], target[2]},
        Vec3{world_up[0], world_up[1], world_up[2]}, fov, width, height);
    const float v[14] = {c.position.x, c.position.y, c.position.z, c.right.x, c.right.y, c.right.z, c.up.x, c.up.y,
        c.up.z, c.forward.x, c.forward.y, c.forward.z, c.fov_scale, c.aspect};
    std::memcpy(out, v, sizeof(v));
}

}  // extern "C"
