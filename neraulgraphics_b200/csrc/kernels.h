// Launch interfaces of the kernels, shared by the host code (renderer.cpp) and the .cu files.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device.cuh"

namespace ngb {

// The tree build of every world, optionally composing the matrices from body poses first.
struct BuildArgs {
    int worlds;
    int per_world;
    long long n;                   // worlds * per_world
    int compose;                   // 0: matrices_in; 1: matrices from body poses; 2: from geom poses
    const float *matrices_in;      // n x 12, when !compose
    const float *body_poses;       // worlds x bodies_per_world x 7, when compose
    const int *body_of_instance;   // per slot
    const float *local_pose;       // per slot, 7
    const float *local_scale;      // per slot, 3
    int bodies_per_world;
    const float *geom_xpos;        // worlds x geoms_per_world x 3, when compose == 2
    const float *geom_xmat;        // worlds x geoms_per_world x 9, when compose == 2
    const int *geom_of_instance;   // per slot, when compose == 2
    const float *geom_scale;       // per slot, 3, when compose == 2
    int geoms_per_world;
    float *matrices_out;           // n x 12, written when compose
    const float *slot_bounds;      // per slot: its mesh's box in mesh space, 6
    const int *slot_blas_root;     // per slot
    float4 *inst;                  // n x 4
    unsigned long long *keys;      // n, instance order
    int *sorted_ids;               // n, sorted order
    float4 *tlas;                  // (2n - 1) x 2
    int *roots;                    // worlds
    int *parent;                   // 2n - 1; parent[0] stays -1
    int *arrivals;                 // n - 1 counters, zero between builds
    int *error_flag;               // set nonzero if a climb runs longer than any valid tree allows
    float4 *tlas_pairs;            // (n - 1) x 4 child-pair records of the internal nodes, or null
    // Worlds of uneven sizes (the per-world build only; per_world is then the largest): world w's instances
    // are [world_first[w], world_first[w + 1]) and the slot tables hold one entry per instance. Null: uniform.
    const int *world_first;
    int *leaf_of;                  // n: each instance's sorted position, or null
};

// Group size (threads per world) of the per-world build: a power of two, at least 32.
int build_group_size(int per_world);
// Largest instance count per world the per-world build handles; above it the global build runs.
constexpr int MAX_PER_WORLD = 1024;
// Largest instance count per world at all: a world's tree is then at most 30 + 22 + 1 deep, which the
// traversal stacks hold (see device.cuh).
constexpr int MAX_INSTANCES_PER_WORLD = 1 << 22;
cudaError_t launch_build_worlds(const BuildArgs &a, cudaStream_t stream);

// The global build: the same tree for any instance count per world, over global memory (see lbvh.cu).
struct LargeBuildScratch {
    float4 *aabb;                   // n x 2: each instance's world box
    int *bounds;                    // worlds x 6: ordered-int centre bounds
    unsigned long long *keys_a;     // n: the radix sort's keys, ping
    unsigned long long *keys_b;     // n: pong
    int *ids_a, *ids_b;             // n each: the ids sorted with them
    unsigned *counts;               // 256 x large_sort_blocks(n)
};
int large_sort_blocks(long long n);
cudaError_t launch_build_large(const BuildArgs &a, const LargeBuildScratch &t, cudaStream_t stream);

// Rendering every view of a batch.
struct RenderArgs {
    const float *cameras;          // views x 12, camera-to-world
    float fov_scale;               // tanf(fov / 2), computed on the host
    float aspect;                  // width / height
    int width;
    int height;                    // the image's height: rays and random streams follow the whole image
    int row_first;                 // the rows rendered, [row_first, row_first + rows) of every view's image;
    int rows;                      // the outputs hold views x rows x W pixels (rows = height: the whole image)
    int cameras_per_world;
    int views;
    int frame;
    int spp;
    uint8_t *rgb;                  // views x rows x W x 3, or null
    float *depth;                  // views x rows x W, or null
    float *normal;                 // views x rows x W x 3, or null
    int32_t *object_id;            // views x rows x W, or null
    int32_t *hit_instance;         // centre ray's hit record, or null
    int32_t *hit_triangle;
    float *hit_u;
    float *hit_v;
    int *error_flag;               // set nonzero if a traversal stack would overflow
    float4 *camera_basis;          // views x 3: scratch for the persistent and tile kernels' per-view camera
    // Per-pixel scratch of the tile kernels, between the camera, shade and shadow kernels (see tiles.cu).
    float4 *pic_hit;               // the picture ray's closest hit: t, u, v, triangle
    int *pic_code;                 // its object code, then the shadowed pixel's bytes
    float4 *shadow_o;              // the shadow ray's origin and length (0: no shadow ray)
    float4 *shadow_d;              // its direction and the lit pixel's bytes
    int *shadow_self;              // the shadow ray's own instance: instance * 4 + mode (1 skip, 2 first), or -1
    // Views of uneven sizes (tile kernels only): per view (width, height, first pixel, first tile), with the
    // totals; null when every view is width x height.
    const int4 *view_info;
    long long total_pixels;
    long long total_tiles;
    // Uneven views: per view its first tile of 4 x 4 pixels, and their total (the camera kernel's paired tiles).
    const int *view_pair_tile;
    long long total_pair_tiles;
    // Single-view renders (Renderer::render / render_frame): camera_basis already holds each view's camera as the
    // caller gave it (no matrix, no renormalising), and the picture's linear radiance per pixel (the average of
    // its samples this frame) goes to radiance instead of bytes to rgb, for launch_accumulate.
    int basis_given;
    float4 *radiance;
    // The tile kernels' per-view candidate order (views x order_stride): instances by the eye's distance to their
    // boxes, and those distances (see tiles.cu view_order_kernel).
    int *view_order;
    float *view_bound;
    int order_stride;
};

// The running average of a single-view renderer's pictures (render_pixel, src/render_core.h:288-301): per pixel
// acc = this frame's radiance with count 1 at frame 0, else the previous acc plus it; the average's sRGB bytes
// as 0xAARRGGBB into argb and, when rgb is not null, as red, green, blue bytes.
cudaError_t launch_accumulate(const float4 *radiance, float4 *accum, int frame, long long pixels, const float *srgb_table,
    uint32_t *argb, uint8_t *rgb, cudaStream_t stream);

// The per-view camera basis of camera_from_matrix (src/render_core.h:264-273): (position.xyz, right.x)
// (right.yz, up.xy) (up.z, forward.xyz) for each view.
cudaError_t launch_prepare_cameras(const float *cameras, int views, float4 *basis, cudaStream_t stream);
cudaError_t launch_render(const SceneParams &s, const RenderArgs &a, cudaStream_t stream);

// Ray queries over the worlds of a batch: ray i belongs to world i / rays_per_world.
struct RayArgs {
    const float *origins;
    const float *directions;
    float max_distance;
    int rays_per_world;
    int count;
    float *distance;
    float *normal;
    int32_t *object_id;
    int *error_flag;
};
cudaError_t launch_rays(const SceneParams &s, const RayArgs &a, cudaStream_t stream);

// The persistent render: spp 1, at most one light, no mirror bounces (see persistent.cu).
struct PersistentTuning {
    int threads;      // per CTA: 64, 128 or 256
    int refill;       // a warp fetches new pixels once this many of its lanes are idle
    int registers;    // register budget per thread: 48, 64 or 72 (not every pair with threads is built)
    int leaf_batch;   // a warp takes a leaf step once this many lanes wait at leaves (or none is at an inner node)
    // The tile kernels' shape: tiles (of 32 rays) a warp takes per fetch, and whether the camera kernel puts a
    // pixel's two rays on adjacent lanes of a 4 x 4 tile (when a render asks for both kinds) or traces 8 x 4 tiles
    // of one kind at a time.
    int tile_fetch = 1;
    int tile_pairs = 1;
};
cudaError_t launch_render_persistent(const SceneParams &s, const RenderArgs &a, int *counter,
    const PersistentTuning &t, cudaStream_t stream);
// Ray queries on the persistent kernel: each lane a ray, refilled from the queue as its walk ends.
cudaError_t launch_rays_persistent(const SceneParams &s, const RayArgs &r, int *counter, const PersistentTuning &t,
    cudaStream_t stream);
// Ray queries as warp packets over each world's tree: 32 consecutive rays of a world per warp (see tiles.cu).
cudaError_t launch_rays_packets(const SceneParams &s, const RayArgs &r, int *counter, cudaStream_t stream);

// The tile render: the persistent kernel's cases, for worlds of at most TILE_MAX_INSTANCES instances (see
// tiles.cu). Of the tuning, threads and registers are read: 128/48, 128/56, 128/64, 128/80 or 256/64.
constexpr int TILE_MAX_INSTANCES = 256;
// after_camera / after_shade (may be null) are recorded on the stream after the camera and shade kernels.
cudaError_t launch_render_tiles(const SceneParams &s, const RenderArgs &a, int *counter, const PersistentTuning &t,
    cudaStream_t stream, cudaEvent_t after_camera, cudaEvent_t after_shade);

// The adjoint of the depth and normal images (see adjoint.cu). Every pointer is device memory; grad_normal
// may be null; the gradients are added to grad_matrices and grad_cameras.
struct AdjointArgs {
    const float *matrices;         // instances x 12: world-from-mesh, as the forward render saw them
    const float *cameras;          // views x 12: camera-to-world
    float fov_scale;
    float aspect;
    int width;
    int height;
    int row_first;                 // the rows the forward rendered (RenderArgs)
    int rows;
    int cameras_per_world;
    int views;
    const int32_t *hit_instance;   // per pixel: the centre ray's hit, -1 for none or not a mesh
    const int32_t *hit_triangle;   // triangle index in its mesh's own list
    const float *hit_u;
    const float *hit_v;
    const float *depth;
    const float *grad_depth;       // per pixel
    const float *grad_normal;      // per pixel, 3, or null
    float *grad_matrices;          // instances x 12
    float *grad_cameras;           // views x 12
    const int *tri_of_local;       // packed triangle of (mesh's first packed triangle + index in its mesh)
    const int *slot_tri_base;      // per slot: its mesh's first packed triangle
};
cudaError_t launch_depth_normal_adjoint(const SceneParams &s, const AdjointArgs &a, cudaStream_t stream);

// A mesh's tree rebuilt on the device from new vertex positions, node for node the host's (see blas_build.cu).
struct MeshBuildArgs {
    const float *vertices;      // vertex_count x 3
    const float *normals;       // vertex_count x 3, or null
    const uint32_t *indices;    // triangles x 3
    int triangles;
    int node_base, tri_base;    // the mesh's first node and first packed triangle
    float4 *blas;               // bvh::Node records, 2 float4 per node
    float4 *pairs;              // child-pair records, 4 float4 per node
    float4 *tris;               // 3 float4 per packed triangle
    float4 *attrs;              // 4 float4 per packed triangle, or null (the scene keeps no normals)
    int *tri_index;             // per packed triangle: its index in the mesh
    int *tri_of_local;          // at tri_base + mesh triangle: its packed index
};
struct MeshBuildScratch {
    float *box;                 // triangles x 6
    float *centre;              // triangles x 3
    uint32_t *order;            // triangles: the leaf order under construction
    int *lpos, *rpos;           // triangles each: a partition's swap positions
    // The tree's nodes in level order (at most 2 triangles - 1).
    float *node_box;            // 6 per node
    int *begin, *end;           // per node: its range of the order
    int *left;                  // per node: its first child (the second follows), or -1 for a leaf
    int *depth;                 // per node
    int *index;                 // per node: its index in the mesh's tree
    int *counter;               // out: the tree's node count
    int *level_count;           // per depth (MESH_LEVELS + 1): the nodes its parents' splits appended
    int *starts, *top, *prefix; // per order position: internal nodes starting there, the least depth of those,
                                // and the internal nodes starting before it
};
constexpr int MESH_LEVELS = 61;  // depths 0..60: a node at depth 60 is a leaf
// The whole rebuild in one cooperative launch: the tree, its packing, and the slots of this mesh (their root
// reference, box and convexity claim); the node count lands in t.counter.
cudaError_t launch_mesh_build(const MeshBuildArgs &a, const MeshBuildScratch &t, const int *slot_mesh, int slots,
    int mesh, int2 *slot_root, float *slot_bounds, float4 *slot_hull, cudaStream_t stream);

}  // namespace ngb
