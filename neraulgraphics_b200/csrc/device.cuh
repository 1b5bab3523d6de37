// Device-side types and math shared by the kernels (compose + tree build, trace, ray queries).
//
// Arithmetic rules. Every kernel file is compiled with -fmad=false and IEEE division and square root, and
// every expression keeps the reference's operation order (src/geom_dev.h, src/render_core.h,
// src/mesh_dev.h, src/cuda_tlas.cuh), so a hit, a depth or a normal is bit-for-bit what the reference's
// CPU backend computes from the same inputs. normalize is v * (1 / sqrt(v.v)) as the reference's host
// code has it (geom_dev.h:45-51), not rsqrtf. Only sinf, cosf and powf (light sampling, specular, sRGB)
// are CUDA's, within a few ulp of the host's; tan(fov / 2) is computed once on the host.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ngb {

constexpr int MAX_SPHERES = 32;
constexpr int MAX_LIGHTS = 8;
constexpr int OBJECT_NONE = 0;
constexpr int OBJECT_SPHERE = 1;
constexpr int OBJECT_FLOOR = OBJECT_SPHERE + MAX_SPHERES;
constexpr int OBJECT_INSTANCE = OBJECT_FLOOR + 1;

constexpr float NO_HIT = 1e30f;
// Stack depths. A mesh's tree is at most 60 deep (the host builder's limit), so 64 entries hold any
// traversal stack over it. A world's LBVH is at most 30 (Morton bits) + ceil(log2(instances)) + 1 deep
// (equal keys split on their positions), 53 for the largest world allowed (2^22 instances).
constexpr int BLAS_STACK = 64;
constexpr int TLAS_STACK = 64;

// The classic-shading fields of a material (include/neraulgraphics/scene.h:35-41); the physically based
// ones are not read by the batched path.
struct DevMaterial {
    float3 diffuse_color;
    float kd;
    float ks;
    float kr;
    float exponent;
    float pad;
};

struct DevSphere {
    float3 center;
    float radius;
    DevMaterial m;
};

// A light as the reference's device code holds it (src/device_scene.h:223-232, 265-272).
struct DevLight {
    float3 position;
    float intensity;
    float radius;
    float falloff;
    float3 direction;
    float cos_outer;
    float cos_inner;
    float3 color;
};

struct DevPlane {
    float y, hx, zmin, zmax, checker;
    DevMaterial m;
};

// Everything a pixel's trace reads besides its camera and the outputs. Passed by value as a
// __grid_constant__ kernel parameter (constant bank), so warp-uniform reads broadcast.
//
// HBM layout of the scene:
//   blas      every mesh's tree, 2 float4 per node: (lo.xyz, a) (hi.xyz, count) -- bvh::Node
//   tris      3 float4 per triangle in leaf order: v0, e1, e2
//   attrs     4 float4 per triangle (vertex normals), or null
//   inst      4 float4 per instance, world-major: world->mesh rows 0..2 (xyz = linear, w = translation),
//             then (blas_root, slot, 0, 0) as ints
//   tlas      2 float4 per node: (lo.xyz, left) (hi.xyz, right) -- bvh::TlasNode; internal nodes 0..n-2,
//             leaf k = node n-1+k
//   roots     per world, the node that roots its tree
struct SceneParams {
    DevSphere spheres[MAX_SPHERES];
    DevLight lights[MAX_LIGHTS];
    DevPlane floor;
    float3 env_up;
    float3 env_color_up;
    float3 env_color_down;
    float env_intensity;
    float ambient;
    int sphere_count;
    int light_count;
    const float4 *tlas;
    const int *roots;
    const float4 *inst;
    const float4 *blas;
    const float4 *tris;
    const float4 *attrs;
    const int *tri_index;
    const DevMaterial *slot_material;
    int instance_count;        // over all worlds
    int per_world;             // instances per world; the most any world holds when world_first is set
    // Worlds of uneven instance counts: world w's instances are [world_first[w], world_first[w + 1]) and the
    // slot tables (slot_*) hold one entry per instance. Null: world w's are [w per_world, (w + 1) per_world)
    // and the slot tables one entry per slot of a world.
    const int *world_first;
    int blas_node_count;  // caps a mesh-tree walk: a correct walk visits each node at most once
    // Child-pair records (both children's boxes and references in 64 bytes; see host.h and lbvh.cu):
    // every mesh node, and every world's internal LBVH nodes by their Karras index.
    const float4 *blas_pairs;
    const float4 *tlas_pairs;
    const int2 *slot_root;     // per slot: its mesh root's reference (node, 0) or (first triangle, count)
    const float *slot_bounds;  // per slot: its mesh's box in mesh space, 6 floats
    int tlas_internal;         // n - 1: nodes below this index are internal
    const float *srgb_table;   // 256 sRGB byte thresholds made on the host (see host.h: srgb_thresholds)
    // Per slot (per instance for uneven worlds): its mesh's vertex mean in mesh space and, in w, its radius
    // when the mesh is convex, else -1 (host.h: mesh_hull). Per instance: its leaf's position among the sorted
    // leaves (leaf node n - 1 + leaf_of[g]).
    const float4 *slot_hull;
    const int *leaf_of;
    // Per slot (per instance for uneven worlds): a sphere in mesh space holding its mesh (host.h: mesh_sphere), or
    // w = -1 for none (a mesh rebuilt on the device).
    const float4 *slot_sphere;
};

// The first instance of world w, its instance count, and the slot-table entry of its instance g.
__device__ __forceinline__ int world_first_of(const SceneParams &s, int w) {
    return s.world_first ? __ldg(s.world_first + w) : w * s.per_world;
}
__device__ __forceinline__ int world_count_of(const SceneParams &s, int w) {
    return s.world_first ? __ldg(s.world_first + w + 1) - __ldg(s.world_first + w) : s.per_world;
}
__device__ __forceinline__ int table_of(const SceneParams &s, int g, int w) {
    return s.world_first ? g : g - w * s.per_world;
}

// ---------------------------------------------------------------------------------------------- math --

__device__ __forceinline__ float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator-(float3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// 1 / x correctly rounded: the same float as 1.0f / x, by the reciprocal's own rounding sequence.
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
__device__ __forceinline__ float3 normalize(float3 v) { return v * recip(sqrtf(dot(v, v))); }
__device__ __forceinline__ float saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
__device__ __forceinline__ float3 reflect(float3 i, float3 n) { return i - n * (2.0f * dot(i, n)); }
__device__ __forceinline__ float3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }

// PCG hash stream (src/geom_dev.h:114-131).
__device__ __forceinline__ uint32_t pcg_hash(uint32_t x) {
    const uint32_t state = x * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
__device__ __forceinline__ float rand_float(uint32_t &r) {
    r = pcg_hash(r);
    return static_cast<float>(r) * 2.3283064365386963e-10f;
}

// A float as an int ordered like the float (src/cuda_tlas.cuh:27-31).
__device__ __forceinline__ int to_ordered(float f) {
    const int i = __float_as_int(f);
    return i ^ ((i >> 31) & 0x7fffffff);
}
__device__ __forceinline__ float from_ordered(int i) { return __int_as_float(i ^ ((i >> 31) & 0x7fffffff)); }

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

}  // namespace ngb
