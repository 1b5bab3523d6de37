/*
 * ngb.h -- C ABI of the B200-native batched multi-world sensor renderer.
 *
 * One renderer holds world_count worlds. Every world holds the same list of mesh instances, placed
 * differently, and is seen by cameras_per_world cameras of width x height pixels. A camera only sees
 * its own world's instances. This is the drop-in for the reference's batched path:
 *
 *   reference (C++)                                      this ABI
 *   BatchRenderer::BatchRenderer   include/neraulgraphics/batch.h:65-68   ngb_create
 *   detail::make_cuda_backend      src/backend.h:88                       ngb_create
 *   BatchRenderer::set_instance_transforms  batch.h:79, backend.h:62      ngb_set_instance_transforms
 *   BatchRenderer::bind_bodies     batch.h:84, backend.h:63               ngb_bind_bodies
 *   BatchRenderer::set_body_poses  batch.h:90, backend.h:65               ngb_set_body_poses
 *   MJWarpBatchRenderer.update     python/neraulgraphics/mujoco.py:304-314  ngb_bind_geoms / ngb_set_geom_poses
 *   BatchRenderer::render          batch.h:103-104, backend.h:67-68       ngb_render / ngb_render_into
 *   BatchRenderer::render_host     batch.h:105-106                        ngb_render_host
 *   BatchRenderer::cast_rays       batch.h:110-111, backend.h:69-70       ngb_cast_rays
 *   Backend::copy_to_host          backend.h:54                           ngb_copy_to_host
 *   BatchRenderer::last_kernel_ms  batch.h:123, backend.h:83              ngb_last_kernel_ms
 *   BatchRenderer::set_ambient     batch.h:126                            ngb_set_ambient
 *   BatchRenderer::set_environment batch.h:129 (gradient sky only)        ngb_set_environment
 *   accessors                      batch.h:115-122                        ngb_width ... ngb_instances_per_world
 *
 * Every entry point returns a status: NGB_OK, or an error whose message ngb_last_error() gives.
 * Validation runs before any state changes, so a rejected call leaves the renderer as it was
 * (include/neraulgraphics/renderer.h:14-15). The messages of rejected input are the reference's
 * (src/batch.cpp, src/validate.cpp, src/mesh_build.cpp).
 *
 * Pointers marked "in memory" are host pointers for NGB_MEMORY_HOST and CUDA device pointers for
 * NGB_MEMORY_DEVICE. Host input is checked (finite, invertible); device input is trusted, as in the
 * reference (batch.h:75-78). Device input is read on the renderer's stream.
 *
 * Completion: by default every call that launches work waits for it (with a bounded wait, after which
 * it returns NGB_TIMEOUT) before returning, as the reference does. ngb_set_sync(h, 0, ...) makes calls
 * stream-ordered instead: they return once the work is queued on the renderer's stream; a host input
 * in pinned memory must then stay unchanged until the stream has passed the call.
 *
 * Calls on one renderer are serialised by a lock of its own; the calling thread's current CUDA device is
 * left as it was.
 *
 * All types here are plain C: no CUDA or C++ types cross this boundary.
 */
#ifndef NGB_H
#define NGB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define NGB_OK 0
#define NGB_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference */
#define NGB_CUDA_ERROR 2       /* neraulgraphics::CudaError (include/neraulgraphics/renderer.h:32-39) */
#define NGB_TIMEOUT 3          /* a bounded wait on the device ran out */
#define NGB_LOGIC_ERROR 4      /* std::logic_error: a null or destroyed renderer (src/batch.cpp:81-89) */

/* Where an array lives (include/neraulgraphics/renderer.h:49). */
#define NGB_MEMORY_HOST 0
#define NGB_MEMORY_DEVICE 1

/* Which images render() produces (include/neraulgraphics/renderer.h:53-58). */
#define NGB_OUTPUT_RGB 1u
#define NGB_OUTPUT_DEPTH 2u
#define NGB_OUTPUT_NORMAL 4u
#define NGB_OUTPUT_OBJECT_ID 8u

/* Object IDs (include/neraulgraphics/scene.h:19-22). */
#define NGB_MAX_SPHERES 32
#define NGB_MAX_LIGHTS 8
#define NGB_OBJECT_NONE 0
#define NGB_OBJECT_SPHERE 1
#define NGB_OBJECT_FLOOR (NGB_OBJECT_SPHERE + NGB_MAX_SPHERES)
#define NGB_OBJECT_INSTANCE (NGB_OBJECT_FLOOR + 1)

typedef struct {
    float x, y, z;
} ngb_vec3;

/* Same fields, order and meaning as neraulgraphics::Material (include/neraulgraphics/scene.h:35-56). */
typedef struct {
    ngb_vec3 diffuse_color;
    float diffuse_albedo;
    float specular_albedo;
    float reflectivity;
    float specular_exponent;
    float roughness;
    float metallic;
    ngb_vec3 emission;
    float transmission;
    float ior;
} ngb_material;

/* neraulgraphics::Sphere (scene.h:63-67). */
typedef struct {
    ngb_vec3 center;
    float radius;
    ngb_material material;
} ngb_sphere;

/* neraulgraphics::Light (scene.h:82-92). */
typedef struct {
    ngb_vec3 position;
    float intensity;
    float radius;
    float falloff;
    ngb_vec3 direction;
    float spot_angle;
    float spot_softness;
    ngb_vec3 color;
} ngb_light;

/* neraulgraphics::Plane (scene.h:96-103). half_extent_x 0 is no floor. */
typedef struct {
    float y;
    float half_extent_x;
    float z_min;
    float z_max;
    float checker_scale;
    ngb_material material;
} ngb_plane;

/* neraulgraphics::Mesh (include/neraulgraphics/mesh.h:160-171) without uvs: vertex_count x 3 floats,
 * index_count uint32 (3 per triangle), and optionally vertex_count x 3 normals (NULL for none). */
typedef struct {
    const float *vertices;
    int32_t vertex_count;
    const uint32_t *indices;
    int32_t index_count;
    const float *normals;
} ngb_mesh;

/* neraulgraphics::Instance (mesh.h:207-222) without textures. transform: the top three rows of the
 * 4x4, row-major (mesh.h:193-198). */
typedef struct {
    int32_t mesh;
    float transform[12];
    ngb_material material;
} ngb_instance;

/* The gradient sky of neraulgraphics::Environment (scene.h:109-121); maps are not supported. */
typedef struct {
    ngb_vec3 up;
    ngb_vec3 color_up;
    ngb_vec3 color_down;
    float intensity;
} ngb_environment;

/* Everything BatchRenderer's constructor takes (batch.h:65-68), as plain data. */
typedef struct {
    int32_t width;
    int32_t height;
    int32_t world_count;
    int32_t cameras_per_world;
    const ngb_sphere *spheres;
    int32_t sphere_count;
    const ngb_light *lights;
    int32_t light_count;
    ngb_plane floor;
    const ngb_mesh *meshes;
    int32_t mesh_count;
    const ngb_instance *instances; /* what one world holds */
    int32_t instance_count;
    int32_t device; /* CUDA device ordinal */
} ngb_scene;

/* neraulgraphics::BatchFrame (batch.h:27-37): the renderer's own buffers, valid until the next render. */
typedef struct {
    int32_t memory;
    int32_t device_id;
    int32_t views;
    int32_t width;
    int32_t height;           /* the rows drawn: the image's height unless ngb_set_rows chose fewer */
    const uint8_t *rgb;
    const float *depth;
    const float *normal;
    const int32_t *object_id;
} ngb_batch_frame;

/* neraulgraphics::RayHits (renderer.h:88-95): the renderer's own buffers, valid until the next ray query. */
typedef struct {
    int32_t memory;
    int32_t device_id;
    int32_t count;
    const float *distance;
    const float *normal;
    const int32_t *object_id;
} ngb_ray_hits;

/* neraulgraphics::Camera (include/neraulgraphics/scene.h:125-132): the single-view renderer's camera, used as
 * given: an eye, a right / up / forward basis, tan(fov / 2) and width / height. */
typedef struct {
    ngb_vec3 position;
    ngb_vec3 right;
    ngb_vec3 up;
    ngb_vec3 forward;
    float fov_scale;
    float aspect;
} ngb_camera;

typedef struct ngb_renderer ngb_renderer;

/* ---- lifetime -------------------------------------------------------------------------------------- */

/* Builds the meshes' trees on the host, uploads them, and places every world's instances where the
 * scene says. Replaces BatchRenderer::BatchRenderer (src/batch.cpp:47-75) with Device::Cuda and
 * CudaBackend::CudaBackend (src/cuda_backend.cu:327-363). On failure *out is NULL and
 * ngb_last_error(NULL) says why. */
int ngb_create(const ngb_scene *scene, ngb_renderer **out);
void ngb_destroy(ngb_renderer *r);

/* The message of the last failed call on r, or of the last failed ngb_create on this thread when r is
 * NULL. Empty after a success. */
const char *ngb_last_error(const ngb_renderer *r);

/* ---- placing the instances ------------------------------------------------------------------------- */

/* world_count * instances_per_world matrices of 12 floats, world-major, in memory. Rebuilds every
 * world's tree over its instances on the GPU. Replaces BatchRenderer::set_instance_transforms
 * (src/batch.cpp:91-109) and CudaBackend::set_instance_matrices (src/cuda_backend.cu:457-469). */
int ngb_set_instance_transforms(ngb_renderer *r, const float *matrices, int32_t memory);

/* How simulator bodies carry the instances: per instance of a world, its body (-1 for none), its pose
 * on the body (x, y, z, qx, qy, qz, qw) and its scale (x, y, z). Host arrays. Replaces
 * BatchRenderer::bind_bodies (src/batch.cpp:111-129, src/cuda_backend.cu:472-491). */
int ngb_bind_bodies(ngb_renderer *r, int32_t bodies_per_world, const int32_t *body_of_instance, const float *local_pose,
    const float *scale);

/* world_count * bodies_per_world poses of 7 floats, world-major, in memory. Composes every instance's
 * matrix and rebuilds the trees, in one launch. Replaces BatchRenderer::set_body_poses
 * (src/batch.cpp:131-144) and CudaBackend::set_body_poses (src/cuda_backend.cu:493-507). */
int ngb_set_body_poses(ngb_renderer *r, const float *body_poses, int32_t memory);

/* How a MuJoCo (or MuJoCo Warp) model's geoms carry the instances: per instance of a world, its geom index
 * in [0, geoms_per_world) and its scale (x, y, z). Host arrays. Replaces the geom list and scales that
 * MJWarpBatchRenderer keeps (python/neraulgraphics/mujoco.py:199-243). Replaces a body binding. */
int ngb_bind_geoms(ngb_renderer *r, int32_t geoms_per_world, const int32_t *geom_of_instance, const float *scale);

/* Every geom's world position and rotation as a simulator's data holds them: geom_xpos world_count x
 * geoms_per_world x 3 floats and geom_xmat world_count x geoms_per_world x 9 floats (row-major 3x3), world-major,
 * both in memory. Each instance's matrix is [R * diag(scale) | p] of its geom, composed inside the tree build's
 * launch: the same matrices as MJWarpBatchRenderer's compose kernel followed by set_instance_transforms
 * (python/neraulgraphics/mujoco.py:287-314), without that kernel or the matrices' round trip through memory. */
int ngb_set_geom_poses(ngb_renderer *r, const float *geom_xpos, const float *geom_xmat, int32_t memory);

/* ---- meshes whose vertices move ----------------------------------------------------------------------- */

/* New vertex positions for mesh `mesh` (the vertex count and triangles it was made with): vertex_count x 3
 * floats in memory, and optionally new vertex normals (NULL keeps the ones it has; a mesh made without normals
 * takes none). The mesh's tree is rebuilt on the device -- the binned SAH build ngb_create runs on the host
 * (src/bvh.cpp:46-174, src/mesh_build.cpp:91-157), node for node -- its triangles re-packed, and every world's
 * instance tree rebuilt from the current transforms. Host arrays are checked as ngb_create checks meshes.
 * No counterpart in the reference, where a mesh changes only by making a new renderer. Waits for the rebuild
 * (it reads each tree level's size back). */
int ngb_update_mesh(ngb_renderer *r, int32_t mesh, const float *vertices, const float *normals, int32_t memory);

/* Mesh `mesh`'s tree as the renderer holds it, in ngb_build_meshes's format for that one mesh (mesh-local
 * node and triangle references): call with NULL arrays for the counts, then with node_count x 8 words,
 * triangle_count x 12 floats, 6 bounds and triangle_count original triangle indices (any may be NULL). */
int ngb_inspect_mesh(ngb_renderer *r, int32_t mesh, int32_t *node_count, int32_t *triangle_count, int32_t *nodes,
    float *triangles, float *bounds, int32_t *triangle_index);

/* ---- rendering ------------------------------------------------------------------------------------- */

/* Renders every view into the renderer's own device buffers, described in *out. view_count cameras of
 * 12 floats (camera-to-world, OpenGL convention) in camera_memory. Replaces BatchRenderer::render
 * (src/batch.cpp:146-162) and CudaBackend::render_batch (src/cuda_backend.cu:509-545). */
int ngb_render(ngb_renderer *r, const float *camera_matrices, float fov, int32_t samples_per_pixel, uint32_t outputs,
    int32_t frame, int32_t camera_memory, ngb_batch_frame *out);

/* The same, writing into caller-owned device buffers (views x H x W x {3 u8, 1 f32, 3 f32, 1 i32}); a
 * buffer may be NULL when its output is not asked for. For callers that own the memory, such as a
 * framework's tensors. */
int ngb_render_into(ngb_renderer *r, const float *camera_matrices, float fov, int32_t samples_per_pixel,
    uint32_t outputs, int32_t frame, int32_t camera_memory, uint8_t *rgb, float *depth, float *normal,
    int32_t *object_id);

/* Renders from host cameras and copies the images into caller-owned host buffers. Replaces
 * BatchRenderer::render_host (src/batch.cpp:164-178). */
int ngb_render_host(ngb_renderer *r, const float *camera_matrices, float fov, int32_t samples_per_pixel,
    uint32_t outputs, int32_t frame, uint8_t *rgb, float *depth, float *normal, int32_t *object_id);

/* rays_per_world rays in every world (world-major, 3 floats each), in memory. Replaces
 * BatchRenderer::cast_rays (src/batch.cpp:180-192) and CudaBackend::cast_rays_batch
 * (src/cuda_backend.cu:547-585). */
int ngb_cast_rays(ngb_renderer *r, const float *origins, const float *directions, int32_t rays_per_world,
    float max_distance, int32_t memory, ngb_ray_hits *out);

/* The same, writing into caller-owned device buffers: rays x {1 f32 distance, 3 f32 normal, 1 i32 ID}. */
int ngb_cast_rays_into(ngb_renderer *r, const float *origins, const float *directions, int32_t rays_per_world,
    float max_distance, int32_t memory, float *distance, float *normal, int32_t *object_id);

/* Copies bytes from one of the renderer's device arrays into host memory (src/backend.h:54). */
int ngb_copy_to_host(ngb_renderer *r, const void *src, void *dst, size_t bytes);

/* ---- settings ---------------------------------------------------------------------------------------- */

int ngb_set_ambient(ngb_renderer *r, float ambient);      /* src/batch.cpp:230-233 */
float ngb_ambient(const ngb_renderer *r);
int ngb_set_environment(ngb_renderer *r, const ngb_environment *environment); /* src/batch.cpp:224-227 */
/* Replaces the lights, at most NGB_MAX_LIGHTS, checked as ngb_create checks them; takes effect on the next render
 * (Renderer::set_lights, src/renderer.cpp:139-143). */
int ngb_set_lights(ngb_renderer *r, const ngb_light *lights, int32_t count);

/* The stream every later call queues its work on: a cudaStream_t, or NULL for the renderer's own stream
 * (created non-blocking at ngb_create). CUDA's legacy default stream is named by its handle,
 * cudaStreamLegacy ((void *)0x1), since NULL here means the renderer's own. */
int ngb_set_stream(ngb_renderer *r, void *cuda_stream);
/* synchronous 1: calls wait for their work, at most timeout_seconds (NGB_TIMEOUT after that).
 * synchronous 0: calls return once the work is queued. */
int ngb_set_sync(ngb_renderer *r, int32_t synchronous, double timeout_seconds);
/* How renders run. kernel: 0 automatic (the tile kernels where they apply: one sample per pixel, at most one
 * light, no material with reflectivity >= 1e-3; else the per-pixel kernel), 1 the per-pixel kernel,
 * 2 the persistent kernel where it applies, 3 the tile kernels where the persistent kernel applies (worlds of
 * at most 256 instances through per-tile candidate lists, larger ones walking their tree as a warp packet).
 * Ray queries (ngb_cast_rays), unless ngb_set_ray_kernel chose otherwise, take warp packets in worlds above 256
 * instances (kernel 0 or 3) and else the persistent kernel in a shape of their own (256/64, refill 28, no leaf
 * batching), unless kernel 2 is chosen, whose shape they then take, or kernel 1 (the per-thread ray kernel).
 * With kernel 3 the call sets the tile kernel's shape: threads_per_block and registers as one of 128/48,
 * 128/56, 128/64, 128/80, 256/64 (default 128/56); refill_lanes and leaf_batch are not read.
 * Otherwise it sets the persistent kernel's shape: threads_per_block and registers (the register budget per
 * thread) as one of 128/48, 128/64, 128/72, 256/48, 256/64, 64/64, refill_lanes (1..32: a warp takes new
 * pixels once this many of its lanes are free) and leaf_batch (1..32: lanes at a leaf wait until this many do,
 * or none is at an internal node, before the warp takes a leaf step). Defaults: 0, 128, 28, 72, 16. */
int ngb_set_tuning(ngb_renderer *r, int32_t kernel, int32_t threads_per_block, int32_t refill_lanes, int32_t registers,
    int32_t leaf_batch);

/* The tile kernels' work shape (kernel 0 or 3 of ngb_set_tuning): tiles_per_fetch (1 to 8) tiles of 32 rays a warp
 * takes with one atomic, 32 to 256 rays per fetch (default 1: the finest balance at the end of a launch); paired 1
 * (default): when a render asks for the picture and the centre-ray images, the camera kernel puts each pixel's two
 * rays on adjacent lanes of a 4 x 4 tile, one pass; 0: 8 x 4 tiles of one kind of ray, two passes. The images
 * are the same bit for bit either way. No counterpart in the reference. */
int ngb_set_tile_shape(ngb_renderer *r, int32_t tiles_per_fetch, int32_t paired);

/* Which kernel answers ray queries (ngb_cast_rays): 0 automatic (warp packets for worlds above 256 instances, else
 * as ngb_set_tuning describes), 1 one thread per ray, 2 the persistent kernel (lanes refilled as their rays end),
 * 3 warp packets: 32 consecutive rays of a world per
 * warp walking the world's tree together, each lane entering only what its own ray enters (for rays of one
 * sensor in scan order, such as a LiDAR's beams). The same hits every way, up to which of two equally distant hits
 * is kept. No counterpart in the reference. */
int ngb_set_ray_kernel(ngb_renderer *r, int32_t kernel);

/* How the instance trees are built. mode 0 (default): one fused launch of per-world groups when a world
 * holds at most 1024 instances, else the global build; 1: always the per-world build (at most 1024 instances
 * per world); 2: always the global build (global radix sort, Karras nodes, bottom-up refit over global
 * memory, the reference's steps in cuda_tlas.cuh:215-306). Both make the same tree. No counterpart in the
 * reference, which always runs its global build. */
int ngb_set_build(ngb_renderer *r, int32_t mode);

/* Bytes of device memory held by every renderer of the process (their device arrays; not the caller's). */
int64_t ngb_device_bytes(void);
/* Testing: host-side fault injection. The after-th device allocation from now on, by any renderer (0: the next
 * one), fails as cudaMalloc does for lack of memory: the call that made it returns NGB_CUDA_ERROR ("out of
 * memory"). A renderer under construction is not made and frees all it made; a renderer stays usable (a failed
 * set_* call leaves the previous tree in place, a failed render leaves its outputs unwritten) and keeps the
 * arrays it made before the failure for its next call. after < 0 cancels. No GPU fault is involved. No
 * counterpart in the reference. */
int ngb_inject_allocation_failure(int32_t after);

/* The rows every later render draws: image rows [first, first + count) of every view, count >= 1 and
 * first + count <= height; (0, height) is the whole image again (the default). The rays, their random streams
 * and so every pixel are the whole image's; the outputs (and ngb_pixel_count, the hit records and the
 * adjoint's per-pixel inputs) hold views x count x width pixels, the band's rows in order. For splitting one
 * large picture across GPUs by rows. Not for worlds of uneven sizes. No counterpart in the reference, which
 * renders whole images. */
int ngb_set_rows(ngb_renderer *r, int32_t first, int32_t count);
/* The rows set by ngb_set_rows: *first and *count (the whole image: 0 and height). */
int ngb_rows(const ngb_renderer *r, int32_t *first, int32_t *count);

/* Waits for every call queued so far, at most timeout_seconds, and reports a kernel's error flag (a
 * traversal stack or walk that ran past what a valid tree allows) as NGB_CUDA_ERROR. */
int ngb_synchronize(ngb_renderer *r, double timeout_seconds);

/* ---- accessors (batch.h:115-123) ------------------------------------------------------------------- */

int32_t ngb_width(const ngb_renderer *r);
int32_t ngb_height(const ngb_renderer *r);
int32_t ngb_world_count(const ngb_renderer *r);
int32_t ngb_cameras_per_world(const ngb_renderer *r);
int32_t ngb_view_count(const ngb_renderer *r);
int32_t ngb_instances_per_world(const ngb_renderer *r);
/* GPU time of the last render or ray query, from CUDA events around its launch (cuda_backend.cu:537-543). */
float ngb_last_kernel_ms(const ngb_renderer *r);
/* The last render's GPU time by kernel, from CUDA events between its launches: *count = 3 for the tile
 * kernels (camera rays, shading, shadow rays), 1 for the others (the whole launch). Up to capacity entries are
 * written. No counterpart in the reference, which times the render as one launch. */
int ngb_last_stage_ms(ngb_renderer *r, float *ms, int32_t capacity, int32_t *count);

/* ---- one view: the single-view Renderer ------------------------------------------------------------- */

/* A renderer made by ngb_create with world_count 1 and cameras_per_world 1 serves as the reference's single-view
 * Renderer (include/neraulgraphics/renderer.h:135-277): its instances move with ngb_set_instance_transforms, its
 * ray queries are ngb_cast_rays with rays_per_world the ray count, and these calls render its view. */

/* A camera at position looking at target, fov the vertical field of view in radians (make_camera,
 * src/renderer.cpp:39-59: the basis in double, then rounded). */
int ngb_make_camera(ngb_vec3 position, ngb_vec3 target, ngb_vec3 world_up, float fov, int32_t width, int32_t height,
    ngb_camera *out);

/* Renderer::render (src/renderer.cpp:104-108; src/cuda_backend.cu:365-374, 642-655): the picture of
 * samples_per_frame jittered rays per pixel, averaged with the frames before it (frame 0 starts the average
 * afresh; frame k > 0 adds its samples to it), as 0xAARRGGBB pixels (alpha 0xFF, gamma-encoded), rows top to
 * bottom, copied into the caller's host buffer argb (width x height; the rows drawn, ngb_set_rows). Waits for the
 * work. Checks as the reference (src/validate.cpp:82-89). */
int ngb_render_view(ngb_renderer *r, const ngb_camera *camera, int32_t frame, int32_t samples_per_frame,
    uint32_t *argb);

/* Renderer::render_frame (src/renderer.cpp:174-182; src/cuda_backend.cu:376-407): the images asked for in the
 * renderer's own device buffers, described in *out (views 1): RGB the running average's bytes (the picture of
 * ngb_render_view, which it also advances), depth, normals and IDs from one ray through each pixel's middle. */
int ngb_render_view_frame(ngb_renderer *r, const ngb_camera *camera, int32_t frame, int32_t samples_per_frame,
    uint32_t outputs, ngb_batch_frame *out);

/* The last view render's 0xAARRGGBB pixels in the renderer's device memory (valid until the next view render):
 * for a caller that shows the picture from the GPU. No counterpart in the reference, whose render copies them. */
int ngb_view_pixels(ngb_renderer *r, const uint32_t **argb);

/* ---- worlds of uneven sizes ------------------------------------------------------------------------- */

/* One world of an uneven batch: its image (its one camera's) and how many instances it holds. */
typedef struct ngb_uneven_world {
    int32_t width;
    int32_t height;
    int32_t instance_count;   /* 0 to 256 */
} ngb_uneven_world;

/* Worlds of uneven instance counts and image sizes in one renderer, rendered by one launch of each tile
 * kernel. scene gives what the worlds share (spheres, lights, floor, meshes, device) and every world's
 * instances, world after world: scene->instances holds the sum of the worlds' instance_count entries, and
 * scene->instance_count that sum; scene->width, height, world_count and cameras_per_world are not read.
 * Matrices (ngb_set_instance_transforms) follow the same order. Renders take one camera per world and need one
 * sample per pixel, at most one light and no reflective material; their images are packed world after world,
 * each world's width x height pixels row-major (ngb_pixel_count in all). Body bindings are not supported.
 * No counterpart in the reference, whose worlds all hold the same instances at one image size. */
int ngb_create_uneven(const ngb_scene *scene, const ngb_uneven_world *worlds, int32_t world_count, ngb_renderer **out);
/* Pixels of one image of every view: views x width x height (height: the rows drawn, ngb_set_rows), or the
 * uneven worlds' sum. */
int64_t ngb_pixel_count(const ngb_renderer *r);

/* ---- differentiation ------------------------------------------------------------------------------- */

/* Copies the last render's hit records (ngb_record_hits) into device arrays of view_count x height x width:
 * the centre ray's instance (-1 when it hit no mesh), its triangle in its mesh's own list, and barycentrics.
 * Any pointer may be NULL. No counterpart in the reference. */
int ngb_copy_hits(ngb_renderer *r, int32_t *instance, int32_t *triangle, float *u, float *v);

/* The adjoint of the depth and normal images: adds d(loss)/d(instance matrices) to grad_matrices (world-major,
 * 12 floats each, the layout of ngb_set_instance_transforms) and d(loss)/d(cameras) to grad_cameras (12 floats
 * per view), given d(loss)/d(depth) (grad_depth, one float per pixel) and d(loss)/d(normals) (grad_normal, 3
 * per pixel, or NULL). Visibility is held fixed: each pixel's recorded hit (from ngb_copy_hits after a render
 * with hit records on) moves with its instance, and the camera rays move with the cameras. matrices, cameras,
 * fov and depth must be those of that render. Every pointer is device memory. No counterpart in the
 * reference, which has no derivatives. */
/* Instance matrices [R(q) diag(s) | p] (12 floats each, q normalised first) of count poses: positions (3
 * floats), quaternions (x, y, z, w) and scales (3 floats, or NULL for 1), all in device memory, queued on
 * `stream` (a cudaStream_t). The matrices of ngb_depth_normal_adjoint's gradient go back to the poses through
 * ngb_pose_matrices_grad: d(loss)/d(positions, quaternions, scales) from d(loss)/d(matrices) (grad_scales may be
 * NULL). No counterpart in the reference; errors: ngb_last_error(NULL). */
int ngb_pose_matrices(const float *positions, const float *quaternions, const float *scales, int64_t count,
    float *matrices, void *stream);
int ngb_pose_matrices_grad(const float *quaternions, const float *scales, int64_t count, const float *grad_matrices,
    float *grad_positions, float *grad_quaternions, float *grad_scales, void *stream);

int ngb_depth_normal_adjoint(ngb_renderer *r, const float *matrices, const float *cameras, float fov,
    const int32_t *hit_instance, const int32_t *hit_triangle, const float *hit_u, const float *hit_v, const float *depth,
    const float *grad_depth, const float *grad_normal, float *grad_matrices, float *grad_cameras);

/* ---- inspection, for parity checks ------------------------------------------------------------------ */

/* Copies the last tree build to host arrays (any may be NULL): the sort keys (world << 32 | Morton
 * code) in instance order, the instance ids in sorted order, the 2n-1 nodes as 8 words each (lo xyz,
 * left, hi xyz, right: the layout of bvh::TlasNode, src/bvh.h:44-49), the per-world roots, and the
 * instance matrices (12 floats each). n = world_count * instances_per_world. */
int ngb_inspect_tlas(ngb_renderer *r, uint64_t *keys, int32_t *sorted_ids, int32_t *nodes, int32_t *roots,
    float *matrices);

/* on 1: later renders that ask for depth, normals or IDs also record each centre ray's hit (see
 * ngb_inspect_hits). Off by default: it writes 16 more bytes per pixel. */
int ngb_record_hits(ngb_renderer *r, int32_t on);

/* Like ngb_record_hits(r, 1), but later renders write the hit records into the caller's device arrays (each
 * view_count x height x width: instance, triangle, u, v; all four given) instead of the renderer's own, saving
 * ngb_copy_hits' copy; ngb_record_hits (either value) goes back to the renderer's own. The arrays must stay
 * valid while renders may write them. No counterpart in the reference. */
int ngb_record_hits_into(ngb_renderer *r, int32_t *instance, int32_t *triangle, float *u, float *v);

/* Per pixel of the last render's centre (depth/normal/ID) rays: the instance hit (over all worlds, -1
 * for none), the triangle hit (its index in its mesh's own list, -1 for none) and the barycentrics u, v.
 * Host arrays of view_count * height * width; any may be NULL. Filled by renders made with
 * ngb_record_hits on that asked for NGB_OUTPUT_DEPTH, NGB_OUTPUT_NORMAL or NGB_OUTPUT_OBJECT_ID. */
int ngb_inspect_hits(ngb_renderer *r, int32_t *instance, int32_t *triangle, float *u, float *v);

/* The 256 sRGB byte thresholds the renderer uses (host only): thresholds[k] is the smallest float whose sRGB
 * byte, (uint8)(saturate(srgb(saturate(v))) * 255 + 0.5) with the host's powf (src/geom_dev.h:169-182), is k
 * or more; thresholds[0] = 0. */
int ngb_srgb_thresholds(float *thresholds);

/* The meshes' bottom-level trees exactly as ngb_create builds them, on the host only (no GPU needed): call
 * with NULL arrays for the counts, then with arrays of node_count x 8 words (bvh::Node: lo xyz, a,
 * hi xyz, count), triangle_count x 12 floats (v0, e1, e2 padded to 4), mesh_count roots,
 * mesh_count x 6 bounds and triangle_count original triangle indices. Errors: ngb_last_error(NULL). */
int ngb_build_meshes(const ngb_mesh *meshes, int32_t mesh_count, int32_t *node_count, int32_t *triangle_count,
    int32_t *nodes, float *triangles, int32_t *roots, float *bounds, int32_t *triangle_index);

/* ---- a tree build that allocates nothing ------------------------------------------------------------- */

/* No counterpart in the reference. The per-world instance-tree build of ngb_set_instance_transforms, for
 * callers that cannot call cudaMalloc, such as a framework whose own pool holds the GPU's memory. Inputs and
 * outputs are the caller's device buffers:
 * matrices (world_count * P * 12 floats), per slot its mesh's box in mesh space (P * 6) and its mesh's
 * BLAS root (P); out: instance records (n * 16 floats: three world->mesh rows, then blas_root and slot as
 * int bits), keys (n), sorted_ids (n), tlas_nodes ((2n - 1) * 8 words, bvh::TlasNode) and roots
 * (world_count), with n = world_count * P. instance_records and tlas_nodes must be 16-byte aligned.
 * Queued on `stream` (a cudaStream_t; NULL is the default stream), not waited for.
 * The build's scratch lives in a static device array of the library: at most 65536 instances over all
 * worlds (and 1024 per world); larger calls return NGB_INVALID_ARGUMENT. Every GPU that loads the library
 * keeps that array (about 0.8 MB) until exit. The first call in a CUDA context (and the first after the
 * calling thread's current context changed, as after cudaDeviceReset) looks up the array's address on the
 * host. All calls share the array: calls that overlap on the GPU race.
 * error_word (device memory, 4-byte aligned, or NULL): set to 0 by the call's work on the stream, then to a
 * nonzero code if the build's bottom-up box climb ran past the step limit a valid tree allows (3: within a
 * world, 4: between worlds), which leaves the tree malformed. Read it once the stream has passed the call. */
int ngb_build_tlas_noalloc(int32_t world_count, int32_t instances_per_world, const float *matrices,
    const float *slot_bounds, const int32_t *slot_blas_root, float *instance_records, uint64_t *keys,
    int32_t *sorted_ids, float *tlas_nodes, int32_t *roots, int32_t *error_word, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NGB_H */
