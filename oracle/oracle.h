/*
 * TEST INFRASTRUCTURE ONLY -- the oracle. Never linked by the product.
 *
 * A CPU restatement, in plain C, of the reference's batched sensor-rendering path (neraulgraphics 0.5.0):
 *   - the meshes' bottom-level trees: binned-SAH build and triangle packing (src/bvh.cpp:46-174,
 *     src/mesh_build.cpp:91-157);
 *   - body poses to instance matrices, in single precision as the reference's GPU does it
 *     (src/cuda_backend.cu:165-202);
 *   - the per-world top-level LBVH of the reference's GPU builder (src/cuda_tlas.cuh:27-211): Morton keys,
 *     stable sort, Karras radix tree, bottom-up boxes, per-world roots;
 *   - the two-level traversal, intersection, shading and the depth/normal/ID images
 *     (src/mesh_dev.h:58-262, src/render_core.h:64-349, src/device_scene.h:98-119, src/geom_dev.h).
 *
 * Arithmetic is IEEE single precision in source order with no fused multiply-adds (built with
 * -ffp-contract=off), which is what the reference's CPU backend computes. Its pins: the reference's
 * own CPU backend and host helpers, compiled from the reference's sources into oracle/_ref/, and the
 * known answers of the reference's tests (tests/test_batch.cpp).
 */
#ifndef NGB_ORACLE_H
#define NGB_ORACLE_H

#include <stdint.h>
#include "../include/ngb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_scene orc_scene;

/* Per-pixel tie flags of orc_render. */
#define ORC_TIE_AOV_INSTANCE 1 /* the centre ray's two nearest hits (different objects) lie within 1e-6 relative t */
#define ORC_TIE_AOV_TRIANGLE 2 /* the centre ray's hit triangle has a neighbour within 1e-6 relative t */
#define ORC_TIE_RGB_INSTANCE 4 /* a jittered primary ray has two objects within 1e-6 relative t */

orc_scene *orc_create(const ngb_scene *scene, char *error, int error_len);
void orc_destroy(orc_scene *s);

/* Host matrices, world-major, 12 floats each: rebuilds the LBVH. */
int orc_set_instance_transforms(orc_scene *s, const float *matrices);
int orc_bind_bodies(orc_scene *s, int bodies_per_world, const int32_t *body_of_instance, const float *local_pose,
    const float *scale);
/* Composes the matrices in single precision (src/cuda_backend.cu:176-202), then rebuilds the LBVH. */
int orc_set_body_poses(orc_scene *s, const float *poses);
void orc_set_ambient(orc_scene *s, float ambient);
void orc_set_environment(orc_scene *s, const ngb_environment *env);

/* Renders every view. Any output pointer may be NULL. hit_*: the centre ray's record (global instance,
 * triangle index in its mesh's own list, barycentrics). ties: ORC_TIE_* per pixel. threads <= 0: all. */
int orc_render(orc_scene *s, const float *cameras, float fov, int spp, unsigned outputs, int frame, uint8_t *rgb,
    float *depth, float *normal, int32_t *ids, int32_t *hit_instance, int32_t *hit_triangle, float *hit_u,
    float *hit_v, uint8_t *ties, int threads);

/* Ray queries, world-major (src/render_core.h:331-349). */
int orc_cast_rays(orc_scene *s, const float *origins, const float *directions, int rays_per_world,
    float max_distance, float *distance, float *normal, int32_t *ids);

/* The last LBVH build: keys in instance order, sorted ids, nodes (8 words each), roots, matrices. */
int orc_tlas(const orc_scene *s, uint64_t *keys, int32_t *sorted_ids, int32_t *nodes, int32_t *roots, float *matrices);
/* The single-view Renderer's render / render_frame for a scene of one world and one camera: camera = position,
 * right, up, forward (3 floats each), fov_scale, aspect, used as given; accum (4 floats per pixel) carries the
 * running average between calls (frame 0 starts it); argb receives the average's 0xAARRGGBB pixels and rgb its
 * bytes; depth, normals, IDs and near-tie flags as orc_render. */
int orc_render_view(orc_scene *s, const float *camera, int spp, unsigned outputs, int frame, float *accum,
    uint32_t *argb, uint8_t *rgb, float *depth, float *normal, int32_t *ids, uint8_t *ties, int threads);

/* The meshes' built trees: counts, then nodes (8 words each), packed triangles (12 floats), per-mesh roots and
 * bounds (6 floats), and each packed triangle's index in its own mesh. */
void orc_blas(const orc_scene *s, int *node_count, int *triangle_count, int32_t *nodes, float *triangles,
    int32_t *roots, float *bounds, int32_t *triangle_index);

/* Bytes the last orc_render's rays fetched while traversing, counted per the rule: 32 per node visited,
 * 64 per pair of child boxes tested, 48 per instance entered, 48 per triangle tested. rays: the rays traced. */
void orc_traversal_bytes(const orc_scene *s, double *bytes, double *rays);

/* Scans the sRGB byte (src/geom_dev.h:169-176, render_core.h:280) of every float in [0, 1]: the number of
 * decreases, and the first float reaching each byte. */
long long orc_srgb_scan(float *first);

/* Single-precision compose alone (src/cuda_backend.cu:165-202), for pinning the GPU compose kernel. */
void orc_compose(int worlds, int per_world, int bodies_per_world, const int32_t *body_of_instance,
    const float *local_pose, const float *scale, const float *poses, float *matrices);

#ifdef __cplusplus
}
#endif

#endif
