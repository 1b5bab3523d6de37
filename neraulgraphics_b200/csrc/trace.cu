// The fused trace-and-shade kernel for every pixel of every view, and the batched ray query.
//
// Per pixel (src/cuda_backend.cu:81-98 and the render core it inlines): the camera from its matrix; the
// picture from spp jittered rays, each shaded with one shadow ray per light (src/render_core.h:202-283);
// and depth, normal and object ID from one centre ray (src/render_core.h:313-327). Rays walk two levels
// (src/mesh_dev.h:113-227): the world's LBVH over instance boxes, then the instance's mesh tree in mesh
// space. Node, instance and triangle data are read through the read-only path (ld.global.nc): they are
// L2-resident for every workload this path serves.
#include "device.cuh"
#include "kernels.h"

#include "trace_common.cuh"

namespace ngb {
namespace {

using namespace tr;

// Pixel mapping: a CTA of 128 threads covers a 16 x 8 tile as four 8 x 4 warp tiles, so each warp's rays
// start from 32 neighbouring pixels. The grid is one long row of tiles, view-major.
constexpr int TILE_W = 16, TILE_H = 8;

__global__ void __launch_bounds__(128) render_kernel(const __grid_constant__ SceneParams s, const RenderArgs a) {
    const int tiles_x = (a.width + TILE_W - 1) / TILE_W, tiles_y = (a.rows + TILE_H - 1) / TILE_H;
    const int tiles = tiles_x * tiles_y;
    const int view = blockIdx.x / tiles, tile = blockIdx.x % tiles;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x = (tile % tiles_x) * TILE_W + (warp & 1) * 8 + (lane & 7);
    const int y = a.row_first + (tile / tiles_x) * TILE_H + (warp >> 1) * 4 + (lane >> 3);
    if (view >= a.views || x >= a.width || y >= a.row_first + a.rows) return;
    // camera_from_matrix (src/render_core.h:264-273); tan(fov / 2) and the aspect come from the host. A
    // single-view render's camera is used as given.
    float3 position, right, up, forward;
    if (a.basis_given) {
        const float4 b0 = __ldg(a.camera_basis + 3 * view), b1 = __ldg(a.camera_basis + 3 * view + 1);
        const float4 b2 = __ldg(a.camera_basis + 3 * view + 2);
        position = mk3(b0.x, b0.y, b0.z);
        right = mk3(b0.w, b1.x, b1.y);
        up = mk3(b1.z, b1.w, b2.x);
        forward = mk3(b2.y, b2.z, b2.w);
    } else {
        const float *m = a.cameras + 12 * static_cast<size_t>(view);
        float cm[12];
        for (int k = 0; k < 12; ++k) cm[k] = __ldg(m + k);
        position = mk3(cm[3], cm[7], cm[11]);
        right = normalize(mk3(cm[0], cm[4], cm[8]));
        up = normalize(mk3(cm[1], cm[5], cm[9]));
        forward = normalize(mk3(-cm[2], -cm[6], -cm[10]));
    }
    const int world = view / a.cameras_per_world;
    const size_t pix = (static_cast<size_t>(view) * a.rows + (y - a.row_first)) * a.width + x;
    const float fw = static_cast<float>(a.width), fh = static_cast<float>(a.height);
    // camera_ray (src/device_scene.h:114-119).
    auto camera_ray = [&](float px, float py) {
        const float sx = (2.0f * px / fw - 1.0f) * a.fov_scale * a.aspect;
        const float sy = -(2.0f * py / fh - 1.0f) * a.fov_scale;
        return normalize(right * sx + up * sy + forward);
    };
    if (a.rgb) {  // render_pixel_rgb8 / sample_pixel (src/render_core.h:248-283)
        uint32_t rng = pcg_hash(static_cast<uint32_t>(y * a.width + x) ^ pcg_hash(static_cast<uint32_t>(a.frame) + 1u));
        float3 sum = mk3(0.0f, 0.0f, 0.0f);
        for (int sample = 0; sample < a.spp; ++sample) {
            const float jx = rand_float(rng);
            const float jy = rand_float(rng);
            sum = sum + trace(s, world, position, camera_ray(static_cast<float>(x) + jx, static_cast<float>(y) + jy),
                              rng, a.error_flag);
        }
        sum = sum * (1.0f / static_cast<float>(a.spp));
        if (a.radiance) {
            a.radiance[pix] = make_float4(sum.x, sum.y, sum.z, 0.0f);
        } else {
            uint8_t *o = a.rgb + 3 * pix;
            o[0] = srgb_byte(s.srgb_table, sum.x);
            o[1] = srgb_byte(s.srgb_table, sum.y);
            o[2] = srgb_byte(s.srgb_table, sum.z);
        }
    }
    if (a.depth || a.normal || a.object_id || a.hit_instance) {  // aov_pixel (src/render_core.h:313-327)
        const float3 dir = camera_ray(static_cast<float>(x) + 0.5f, static_cast<float>(y) + 0.5f);
        Hit hit;
        const bool found = scene_intersect(s, world, position, dir, hit, a.error_flag);
        if (a.depth) a.depth[pix] = found ? hit.t * dot(dir, forward) : __int_as_float(0x7f800000);
        if (a.normal) {
            const float3 n = found ? hit.normal : mk3(0.0f, 0.0f, 0.0f);
            a.normal[3 * pix] = n.x;
            a.normal[3 * pix + 1] = n.y;
            a.normal[3 * pix + 2] = n.z;
        }
        if (a.object_id) a.object_id[pix] = found ? hit.object : OBJECT_NONE;
        if (a.hit_instance) {
            a.hit_instance[pix] = found ? hit.instance : -1;
            a.hit_triangle[pix] = (found && hit.triangle >= 0) ? __ldg(s.tri_index + hit.triangle) : -1;
            a.hit_u[pix] = found ? hit.u : 0.0f;
            a.hit_v[pix] = found ? hit.v : 0.0f;
        }
    }
}

// One ray of a ray query (src/render_core.h:331-349).
__global__ void __launch_bounds__(128) ray_kernel(const __grid_constant__ SceneParams s, const RayArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const int world = i / a.rays_per_world;
    const float3 o = mk3(__ldg(a.origins + 3 * i), __ldg(a.origins + 3 * i + 1), __ldg(a.origins + 3 * i + 2));
    float3 d = mk3(__ldg(a.directions + 3 * i), __ldg(a.directions + 3 * i + 1), __ldg(a.directions + 3 * i + 2));
    const float len2 = dot(d, d);
    Hit hit;
    bool found = len2 > 1e-30f && len2 < 1e30f;
    if (found) {
        d = d * (1.0f / sqrtf(len2));
        found = scene_intersect(s, world, o, d, hit, a.error_flag) && hit.t <= a.max_distance;
    }
    a.distance[i] = found ? hit.t : __int_as_float(0x7f800000);
    const float3 n = found ? hit.normal : mk3(0.0f, 0.0f, 0.0f);
    a.normal[3 * i] = n.x;
    a.normal[3 * i + 1] = n.y;
    a.normal[3 * i + 2] = n.z;
    a.object_id[i] = found ? hit.object : OBJECT_NONE;
}

// One thread per view: the camera basis of camera_from_matrix (src/render_core.h:264-273), renormalised.
__global__ void __launch_bounds__(128) prepare_cameras_kernel(const float *cameras, int views, float4 *basis) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= views) return;
    float m[12];
    for (int k = 0; k < 12; ++k) m[k] = __ldg(cameras + 12 * static_cast<size_t>(v) + k);
    const float3 right = normalize(mk3(m[0], m[4], m[8]));
    const float3 up = normalize(mk3(m[1], m[5], m[9]));
    const float3 fwd = normalize(mk3(-m[2], -m[6], -m[10]));
    basis[3 * v] = make_float4(m[3], m[7], m[11], right.x);
    basis[3 * v + 1] = make_float4(right.y, right.z, up.x, up.y);
    basis[3 * v + 2] = make_float4(up.z, fwd.x, fwd.y, fwd.z);
}

// One thread per pixel: the running average and its bytes (render_pixel, src/render_core.h:288-301, and
// pack_argb8888, src/geom_dev.h:179-184).
__global__ void __launch_bounds__(256) accumulate_kernel(const float4 *radiance, float4 *accum, int frame,
    long long pixels, const float *srgb_table, uint32_t *argb, uint8_t *rgb) {
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < pixels;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float4 r = radiance[p];
        float4 acc = make_float4(r.x, r.y, r.z, 1.0f);
        if (frame != 0) {
            const float4 prev = accum[p];
            acc = make_float4(prev.x + r.x, prev.y + r.y, prev.z + r.z, prev.w + 1.0f);
        }
        accum[p] = acc;
        const float inv = recip(acc.w);
        const uint32_t red = srgb_byte(srgb_table, acc.x * inv), green = srgb_byte(srgb_table, acc.y * inv);
        const uint32_t blue = srgb_byte(srgb_table, acc.z * inv);
        argb[p] = 0xFF000000u | (red << 16) | (green << 8) | blue;
        if (rgb) {
            rgb[3 * p] = static_cast<uint8_t>(red);
            rgb[3 * p + 1] = static_cast<uint8_t>(green);
            rgb[3 * p + 2] = static_cast<uint8_t>(blue);
        }
    }
}

}  // namespace

cudaError_t launch_accumulate(const float4 *radiance, float4 *accum, int frame, long long pixels, const float *srgb_table,
    uint32_t *argb, uint8_t *rgb, cudaStream_t stream) {
    if (pixels <= 0) return cudaSuccess;
    long long blocks = (pixels + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    accumulate_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(radiance, accum, frame, pixels, srgb_table,
        argb, rgb);
    return cudaGetLastError();
}

cudaError_t launch_render(const SceneParams &s, const RenderArgs &a, cudaStream_t stream) {
    const long long tiles = static_cast<long long>((a.width + TILE_W - 1) / TILE_W) * ((a.rows + TILE_H - 1) / TILE_H);
    const long long blocks = tiles * a.views;
    if (blocks <= 0) return cudaSuccess;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    render_kernel<<<static_cast<unsigned>(blocks), 128, 0, stream>>>(s, a);
    return cudaGetLastError();
}

cudaError_t launch_prepare_cameras(const float *cameras, int views, float4 *basis, cudaStream_t stream) {
    if (views <= 0) return cudaSuccess;
    prepare_cameras_kernel<<<(views + 127) / 128, 128, 0, stream>>>(cameras, views, basis);
    return cudaGetLastError();
}

cudaError_t launch_rays(const SceneParams &s, const RayArgs &a, cudaStream_t stream) {
    if (a.count <= 0) return cudaSuccess;
    ray_kernel<<<(a.count + 127) / 128, 128, 0, stream>>>(s, a);
    return cudaGetLastError();
}

}  // namespace ngb
