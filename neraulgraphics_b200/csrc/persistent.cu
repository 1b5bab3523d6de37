// The persistent render kernel: the batched path's common case (one sample per pixel, at most one light,
// no mirror bounces) with full SIMD lanes.
//
// The first render kernel (trace.cu) gives each thread a pixel and walks its rays one after another, the
// world's tree and a mesh's tree in nested loops; a warp then waits for its slowest lane at every level and
// every ray, and only a quarter of the lanes did work per instruction. Here every lane holds one ray job and
// all jobs share one walk loop:
//   - a pixel gives two jobs, the jittered picture ray and the centre ray of the depth/normal/ID images
//     (two neighbouring lanes trace nearly the same ray); a picture ray that hits a lit surface turns into
//     its shadow ray in the same lane;
//   - warps are persistent: when enough of a warp's lanes are free (ballot), one lane takes that many new jobs
//     from a global counter with one atomic and the free lanes start them (warp-ballot compaction, persistent
//     per-warp ray fetch);
//   - the walk is one loop over both levels: entering an instance pushes a marker and moves the ray to mesh
//     space, popping the marker moves it back, so lanes at different levels run the same instructions;
//   - nodes are child-pair records, both children's boxes and references in 64 bytes (four 16-byte loads
//     instead of the six a node plus its two children cost in the reference's layout).
// The walk order is the reference's exactly (nearer child first by dl <= dr, the farther one pushed with its
// entry distance, dropped at pop time once a hit is closer; src/mesh_dev.h:113-159), over the same boxes, so
// every hit, including which of two tied hits wins, is the reference's. The shading arithmetic is the
// reference's, term by term (src/render_core.h:202-283).
#include <climits>

#include "kernels.h"
#include "trace_common.cuh"

namespace ngb {
namespace {

using namespace tr;

// World tree (<= 30 Morton levels + 22 levels among equal keys + 1 for 2^22 instances) + marker + mesh tree (<= 64).
constexpr int STACK = 128;
constexpr int MARKER = INT_MIN;   // stack entry that returns the walk from a mesh to its world's tree
constexpr int ST_IDLE = 0, ST_WALK = 1, ST_DONE = 2;
constexpr int JOB_RGB = 1, JOB_SHADOW = 2, JOB_AOV = 3, JOB_RAY = 4;
constexpr int KINDS_RAYS = 4;     // a launch of ray queries (cast_rays) instead of views
constexpr unsigned FULL = 0xffffffffu;

// A lane's hot state, in registers: the current ray (world space, or mesh space inside an instance), the
// current node, the stack depth and the closest hit so far.
struct Lane {
    int state, job;
    int world;
    float3 o, d, inv;
    float tmax;
    int ref, count;     // current node: (internal, 0), (instance, -1) or (first triangle, count)
    int sp;
    int inst;
    bool in_blas, any, blocked;
    int hit_inst, hit_tri;
    int steps;
};

// A lane's cold state, in shared memory, one column per thread (structure of arrays, conflict-free): what is
// read only when a walk enters or leaves an instance, records a hit, or ends.
enum Cold {
    C_WO, C_WD = C_WO + 3, C_WINV = C_WD + 3,  // the world-space ray while the walk is inside an instance
    C_HU = C_WINV + 3, C_HV,                   // barycentrics of the closest hit
    C_PIX_LO, C_PIX_HI, C_RNG,
    C_FWD, C_LIT = C_FWD + 3, C_SHADOW = C_LIT + 3,
    C_SPHERE = C_SHADOW + 3, C_FLOOR,
    C_FIELDS
};

struct ColdRef {
    float *base;
    int stride;
    __device__ __forceinline__ float &f(int field) const { return base[field * stride]; }
    __device__ __forceinline__ int &i(int field) const { return reinterpret_cast<int *>(base)[field * stride]; }
    __device__ __forceinline__ void put3(int field, float3 v) const {
        f(field) = v.x;
        f(field + 1) = v.y;
        f(field + 2) = v.z;
    }
    __device__ __forceinline__ float3 get3(int field) const { return mk3(f(field), f(field + 1), f(field + 2)); }
    __device__ __forceinline__ void put_pix(long long p) const {
        i(C_PIX_LO) = static_cast<int>(p & 0xffffffffLL);
        i(C_PIX_HI) = static_cast<int>(p >> 32);
    }
    __device__ __forceinline__ long long pix() const {
        return (static_cast<long long>(i(C_PIX_HI)) << 32) | static_cast<unsigned>(i(C_PIX_LO));
    }
};

// Starts a walk of the world's meshes from the ray in L (o, d) with tmax: the root box test of
// traverse<true> (src/mesh_dev.h:117), then the root itself.
__device__ __forceinline__ void start_walk(const SceneParams &s, Lane &L) {
    L.inv = safe_inverse(L.d);
    L.sp = 0;
    L.in_blas = false;
    L.blocked = false;
    L.hit_inst = -1;
    L.steps = 0;
    if (s.instance_count <= 0) {
        L.state = ST_DONE;
        return;
    }
    const int root = __ldg(s.roots + L.world);
    const float4 r0 = __ldg(s.tlas + 2 * root), r1 = __ldg(s.tlas + 2 * root + 1);
    if (box_entry(r0, r1, L.o, L.inv, L.tmax) >= NO_HIT) {
        L.state = ST_DONE;
        return;
    }
    if (root < s.tlas_internal) {
        L.ref = root;
        L.count = 0;
    } else {
        L.ref = ~__float_as_int(r0.w);  // a world of one instance: its root is that instance's leaf
        L.count = -1;
    }
    L.state = ST_WALK;
}

// The walk's pop (traverse's dead end, src/mesh_dev.h:154-157): resume from the stack, dropping what a closer
// hit has put out of reach; a marker hands the walk back to the world's tree.
__device__ __forceinline__ void walk_pop(Lane &L, const ColdRef &cold, const int4 *st) {
    for (;;) {
        int4 e = make_int4(0, 0, 0, 0);
        while (L.sp > 0) {
            e = st[L.sp - 1];
            if (__int_as_float(e.z) < L.tmax) break;
            --L.sp;
        }
        if (L.sp == 0) {
            L.state = ST_DONE;
            return;
        }
        --L.sp;
        const int c = e.y;
        if (c == MARKER) {
            L.o = cold.get3(C_WO);
            L.d = cold.get3(C_WD);
            L.inv = cold.get3(C_WINV);
            L.in_blas = false;
            continue;
        }
        L.ref = e.x;
        L.count = c;
        return;
    }
}

// A walk step at an internal node of either tree: both children's boxes, the nearer one next, the farther one
// pushed with its entry distance (traverse, src/mesh_dev.h:133-151).
__device__ __forceinline__ void walk_inner(const SceneParams &s, Lane &L, const ColdRef &cold, int4 *st, int *err) {
    const float4 *rec = (L.in_blas ? s.blas_pairs : s.tlas_pairs) + 4 * static_cast<long long>(L.ref);
    const float4 q0 = __ldg(rec), q1 = __ldg(rec + 1), q2 = __ldg(rec + 2), q3 = __ldg(rec + 3);
    const float dl = box_entry(make_float4(q0.x, q0.y, q0.z, 0.0f), make_float4(q0.w, q1.x, q1.y, 0.0f), L.o, L.inv, L.tmax);
    const float dr = box_entry(make_float4(q1.z, q1.w, q2.x, 0.0f), make_float4(q2.y, q2.z, q2.w, 0.0f), L.o, L.inv, L.tmax);
    if (dl < NO_HIT || dr < NO_HIT) {
        const bool left_first = dl <= dr;
        const float far_t = left_first ? dr : dl;
        if (far_t < NO_HIT) {
            if (L.sp >= STACK) {
                *err = 1;
                L.state = ST_DONE;
                return;
            }
            st[L.sp] = make_int4(__float_as_int(left_first ? q3.z : q3.x), __float_as_int(left_first ? q3.w : q3.y),
                __float_as_int(far_t), 0);
            ++L.sp;
        }
        L.ref = __float_as_int(left_first ? q3.x : q3.z);
        L.count = __float_as_int(left_first ? q3.y : q3.w);
        return;
    }
    walk_pop(L, cold, st);
}

// A walk step at a leaf: an instance (into its mesh's space, and its mesh root's box test: blas_walk's first
// line) or one triangle of a mesh leaf, in the leaf's order (mesh_intersect / mesh_occluded's leaves,
// src/mesh_dev.h:180-226).
__device__ __forceinline__ void walk_leaf(const SceneParams &s, Lane &L, const ColdRef &cold, int4 *st, int *err) {
    if (L.count < 0) {
        const InstanceRec r = load_instance(s.inst, L.ref);
        const int slot = __float_as_int(__ldg(s.inst + 4 * L.ref + 3).y);
        const float3 lo = to_local_point(r, L.o);
        const float3 ld = to_local_dir(r, L.d);
        const float3 linv = safe_inverse(ld);
        const float *b = s.slot_bounds + 6 * slot;
        const float4 blo = make_float4(__ldg(b), __ldg(b + 1), __ldg(b + 2), 0.0f);
        const float4 bhi = make_float4(__ldg(b + 3), __ldg(b + 4), __ldg(b + 5), 0.0f);
        if (box_entry(blo, bhi, lo, linv, L.tmax) < NO_HIT) {
            if (L.sp >= STACK) {
                *err = 1;
                L.state = ST_DONE;
                return;
            }
            st[L.sp] = make_int4(MARKER, MARKER, __float_as_int(-INFINITY), 0);  // never dropped by the tmax test
            ++L.sp;
            const int2 root = __ldg(s.slot_root + slot);
            // The world-space ray waits in shared memory while the walk is in mesh space.
            cold.put3(C_WO, L.o);
            cold.put3(C_WD, L.d);
            cold.put3(C_WINV, L.inv);
            L.o = lo;
            L.d = ld;
            L.inv = linv;
            L.inst = L.ref;
            L.in_blas = true;
            L.ref = root.x;
            L.count = root.y;
            return;
        }
    } else {
        const int j = L.ref;
        float t, bu, bv;
        if (triangle_hit(s.tris, j, L.o, L.d, L.tmax, t, bu, bv)) {
            if (L.any) {
                L.blocked = true;
                L.state = ST_DONE;
                return;
            }
            L.tmax = t;
            L.hit_inst = L.inst;
            L.hit_tri = j;
            cold.f(C_HU) = bu;
            cold.f(C_HV) = bv;
        }
        if (L.count > 1) {
            ++L.ref;
            --L.count;
            return;
        }
    }
    walk_pop(L, cold, st);
}

// A new job from its item number. Items run over views, then 4 x 4 pixel tiles, then the pixels of a tile,
// then (when both are asked for) the picture ray and the centre ray of a pixel.
__device__ __forceinline__ void start_job(const SceneParams &s, const RenderArgs &a, const RayArgs &ra, Lane &L,
    const ColdRef &cold, long long item, int kinds, int tiles_x, int tiles_per_view) {
    if (kinds == KINDS_RAYS) {
        // A ray query (cast_ray, src/render_core.h:331-349): the direction normalised, a miss if its length is
        // out of range; spheres and the floor, then the meshes; a hit beyond max_distance is a miss.
        const long long i = item;
        const float3 o = mk3(__ldg(ra.origins + 3 * i), __ldg(ra.origins + 3 * i + 1), __ldg(ra.origins + 3 * i + 2));
        float3 d = mk3(__ldg(ra.directions + 3 * i), __ldg(ra.directions + 3 * i + 1), __ldg(ra.directions + 3 * i + 2));
        const float len2 = dot(d, d);
        if (!(len2 > 1e-30f && len2 < 1e30f)) {
            ra.distance[i] = __int_as_float(0x7f800000);
            ra.normal[3 * i] = ra.normal[3 * i + 1] = ra.normal[3 * i + 2] = 0.0f;
            ra.object_id[i] = OBJECT_NONE;
            L.state = ST_IDLE;
            return;
        }
        d = d * (1.0f / sqrtf(len2));
        L.job = JOB_RAY;
        cold.put_pix(i);
        L.world = static_cast<int>(i / ra.rays_per_world);
        L.o = o;
        L.d = d;
        float best = 1e30f;
        int best_sphere = -1;
        for (int k = 0; k < s.sphere_count; ++k) {
            float t;
            if (sphere_hit(s.spheres[k], o, d, t) && t < best) {
                best = t;
                best_sphere = k;
            }
        }
        bool hit_floor = false;
        float dd;
        if (floor_hit(s.floor, o, d, best, dd)) {
            best = dd;
            hit_floor = true;
        }
        cold.i(C_SPHERE) = best_sphere;
        cold.i(C_FLOOR) = hit_floor ? 1 : 0;
        L.tmax = best;
        L.any = false;
        start_walk(s, L);
        return;
    }
    int job = JOB_RGB;
    if (kinds == 3) {
        job = (item & 1) ? JOB_AOV : JOB_RGB;
        item >>= 1;
    } else if (kinds == 2) {
        job = JOB_AOV;
    }
    const long long per_view = 16LL * tiles_per_view;
    const int view = static_cast<int>(item / per_view);
    const int q = static_cast<int>(item % per_view);
    const int tile = q >> 4, within = q & 15;
    const int x = (tile % tiles_x) * 4 + (within & 3);
    const int y = a.row_first + (tile / tiles_x) * 4 + (within >> 2);
    if (x >= a.width || y >= a.row_first + a.rows) {
        L.state = ST_IDLE;
        return;
    }
    L.job = job;
    cold.put_pix((static_cast<long long>(view) * a.rows + (y - a.row_first)) * a.width + x);
    L.world = view / a.cameras_per_world;
    // The view's camera (camera_from_matrix, src/render_core.h:264-273), made once per view by
    // prepare_cameras: (position.xyz, right.x) (right.yz, up.xy) (up.z, forward.xyz).
    const float4 c0 = __ldcg(a.camera_basis + 3 * view), c1 = __ldcg(a.camera_basis + 3 * view + 1);
    const float4 c2 = __ldcg(a.camera_basis + 3 * view + 2);
    const float3 right = mk3(c0.w, c1.x, c1.y);
    const float3 up = mk3(c1.z, c1.w, c2.x);
    const float3 fwd = mk3(c2.y, c2.z, c2.w);
    const float fw = static_cast<float>(a.width), fh = static_cast<float>(a.height);
    float px = static_cast<float>(x) + 0.5f, py = static_cast<float>(y) + 0.5f;
    if (job == JOB_RGB) {
        uint32_t rng = pcg_hash(static_cast<uint32_t>(y * a.width + x) ^ pcg_hash(static_cast<uint32_t>(a.frame) + 1u));
        const float jx = rand_float(rng);
        const float jy = rand_float(rng);
        cold.i(C_RNG) = static_cast<int>(rng);
        px = static_cast<float>(x) + jx;
        py = static_cast<float>(y) + jy;
    }
    cold.put3(C_FWD, fwd);
    L.o = mk3(c0.x, c0.y, c0.z);
    L.d = camera_dir(right, up, fwd, px, py, fw, fh, a.fov_scale, a.aspect);
    // Spheres and the floor first; the meshes are walked with their closest hit as the limit
    // (scene_intersect, src/render_core.h:78-112).
    float best = 1e30f;
    int best_sphere = -1;
    for (int i = 0; i < s.sphere_count; ++i) {
        float t;
        if (sphere_hit(s.spheres[i], L.o, L.d, t) && t < best) {
            best = t;
            best_sphere = i;
        }
    }
    bool hit_floor = false;
    {
        float dd;
        if (floor_hit(s.floor, L.o, L.d, best, dd)) {
            best = dd;
            hit_floor = true;
        }
    }
    cold.i(C_SPHERE) = best_sphere;
    cold.i(C_FLOOR) = hit_floor ? 1 : 0;
    L.tmax = best;
    L.any = false;
    start_walk(s, L);
}

// What happens when a lane's walk ends: outputs, and for a lit picture hit, its shadow ray.
__device__ __forceinline__ void complete(const SceneParams &s, const RenderArgs &a, const RayArgs &ra, Lane &L,
    const ColdRef &cold) {
    const long long pix = cold.pix();
    if (L.job == JOB_SHADOW) {
        write_rgb(s.srgb_table, a.rgb, pix, cold.get3(L.blocked ? C_SHADOW : C_LIT));
        L.state = ST_IDLE;
        return;
    }
    const bool mesh = L.hit_inst >= 0;
    const int best_sphere = cold.i(C_SPHERE);
    const bool hit_floor = cold.i(C_FLOOR) != 0;
    const bool found = mesh || best_sphere >= 0 || hit_floor;
    float3 normal = mk3(0.0f, 0.0f, 0.0f), point = mk3(0.0f, 0.0f, 0.0f);
    DevMaterial mat{};
    int object = OBJECT_NONE;
    if (found) {  // the surface, as scene_intersect resolves it (src/render_core.h:116-141)
        point = L.o + L.d * L.tmax;
        if (mesh) {
            normal = mesh_surface(s, L.hit_inst, L.hit_tri, cold.f(C_HU), cold.f(C_HV), L.d);
            const int slot = L.hit_inst - L.world * s.per_world;
            mat = s.slot_material[slot];
            object = OBJECT_INSTANCE + slot;
        } else if (hit_floor) {
            object = OBJECT_FLOOR;
            normal = mk3(0.0f, 1.0f, 0.0f);
            mat = s.floor.m;
            const int cx = static_cast<int>(floorf(point.x * s.floor.checker));
            const int cz = static_cast<int>(floorf(point.z * s.floor.checker));
            const float3 tint = ((cx + cz) & 1) ? mk3(1.0f, 1.0f, 1.0f) : mk3(1.0f, 0.7f, 0.3f);
            mat.diffuse_color = tint * 0.3f;
        } else {
            normal = normalize(point - s.spheres[best_sphere].center);
            mat = s.spheres[best_sphere].m;
            object = OBJECT_SPHERE + best_sphere;
        }
    }
    if (L.job == JOB_RAY) {
        const long long i = cold.pix();
        const bool hit = found && L.tmax <= ra.max_distance;
        ra.distance[i] = hit ? L.tmax : __int_as_float(0x7f800000);
        const float3 n = hit ? normal : mk3(0.0f, 0.0f, 0.0f);
        ra.normal[3 * i] = n.x;
        ra.normal[3 * i + 1] = n.y;
        ra.normal[3 * i + 2] = n.z;
        ra.object_id[i] = hit ? object : OBJECT_NONE;
        L.state = ST_IDLE;
        return;
    }
    if (L.job == JOB_AOV) {  // aov_pixel (src/render_core.h:313-327)
        const size_t p = static_cast<size_t>(pix);
        if (a.depth) a.depth[p] = found ? L.tmax * dot(L.d, cold.get3(C_FWD)) : __int_as_float(0x7f800000);
        if (a.normal) {
            a.normal[3 * p] = normal.x;
            a.normal[3 * p + 1] = normal.y;
            a.normal[3 * p + 2] = normal.z;
        }
        if (a.object_id) a.object_id[p] = object;
        if (a.hit_instance) {
            a.hit_instance[p] = mesh ? L.hit_inst : -1;
            a.hit_triangle[p] = mesh ? __ldg(s.tri_index + L.hit_tri) : -1;
            a.hit_u[p] = mesh ? cold.f(C_HU) : 0.0f;
            a.hit_v[p] = mesh ? cold.f(C_HV) : 0.0f;
        }
        L.state = ST_IDLE;
        return;
    }
    // The picture ray (trace, src/render_core.h:202-245, one bounce).
    if (!found) {
        const float t = saturate(dot(L.d, s.env_up) * 0.5f + 0.5f);
        const float3 sky = (s.env_color_down + (s.env_color_up - s.env_color_down) * t) * s.env_intensity;
        write_rgb(s.srgb_table, a.rgb, pix, mk3(0.0f, 0.0f, 0.0f) + sky * 1.0f);
        L.state = ST_IDLE;
        return;
    }
    const float3 zero = mk3(0.0f, 0.0f, 0.0f);
    if (s.light_count == 1) {
        const DevLight &lt = s.lights[0];
        uint32_t rng = static_cast<uint32_t>(cold.i(C_RNG));
        const float z = 1.0f - 2.0f * rand_float(rng);
        const float rad = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        const float phi = 6.28318530718f * rand_float(rng);
        const float3 lp = lt.position + mk3(rad * cosf(phi), rad * sinf(phi), z) * lt.radius;
        const float3 to_light = lp - point;
        const float light_distance = sqrtf(dot(to_light, to_light));
        const float3 light_dir = to_light * (1.0f / light_distance);
        const float strength = lt.intensity * light_factor(lt, light_dir, light_distance);
        if (strength > 0.0f) {
            const float3 lit = lt.color * strength;
            const float3 diffuse = zero + lit * fmaxf(0.0f, dot(light_dir, normal));
            const float3 specular = zero + lit * powf(fmaxf(0.0f, dot(reflect(light_dir, normal), L.d)), mat.exponent);
            const float3 c_shadow = radiance_of(mat, s.ambient, zero, zero);
            const float3 c_lit = radiance_of(mat, s.ambient, diffuse, specular);
            // A shadow ray whose answer cannot change the pixel (lit and shadowed bytes equal, as where the
            // surface faces away from the light and the highlight rounds away) is not traced.
            if (rgb_packed(s.srgb_table, c_lit) == rgb_packed(s.srgb_table, c_shadow)) {
                write_rgb(s.srgb_table, a.rgb, pix, c_shadow);
                L.state = ST_IDLE;
                return;
            }
            cold.put3(C_LIT, c_lit);
            cold.put3(C_SHADOW, c_shadow);
            // The shadow ray: spheres and the floor first, then any hit in the meshes (scene_occluded,
            // src/render_core.h:146-161).
            L.job = JOB_SHADOW;
            L.o = offset_origin(point, normal, light_dir);
            L.d = light_dir;
            L.tmax = light_distance;
            L.any = true;
            bool blocked = false;
            for (int i = 0; i < s.sphere_count && !blocked; ++i) {
                float t;
                if (sphere_hit(s.spheres[i], L.o, L.d, t) && t < light_distance) blocked = true;
            }
            if (!blocked) {
                float dd;
                blocked = floor_hit(s.floor, L.o, L.d, light_distance, dd);
            }
            if (blocked) {
                write_rgb(s.srgb_table, a.rgb, pix, c_shadow);
                L.state = ST_IDLE;
                return;
            }
            start_walk(s, L);
            return;
        }
    }
    write_rgb(s.srgb_table, a.rgb, pix, radiance_of(mat, s.ambient, zero, zero));
    L.state = ST_IDLE;
}

// THREADS per CTA and MIN_BLOCKS resident CTAs per SM set the register budget (65536 / (THREADS * MIN_BLOCKS)):
// the walk's temporaries fit 64 registers without spilling, which doubles the warps per scheduler over the
// compiler's unbounded choice (92).
template <int THREADS, int MIN_BLOCKS>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) render_persistent_kernel(const __grid_constant__ SceneParams s,
    const RenderArgs a, const RayArgs ra, int *counter, long long total, int kinds, int tiles_x, int tiles_per_view,
    int refill, int leaf_batch) {
    extern __shared__ float cold_smem[];
    int4 st[STACK];  // (reference, count, entry distance) per pushed node, stored and loaded whole
    const int lane = threadIdx.x & 31;
    const unsigned lanes_below = (1u << lane) - 1u;
    const ColdRef cold{cold_smem + threadIdx.x, THREADS};
    Lane L;
    L.state = ST_IDLE;
    // A correct walk visits each node of its world's tree once and each node of an entered mesh's tree once.
    const long long cap = 2LL * s.per_world + 2 + static_cast<long long>(s.per_world) * (s.blas_node_count + 2);
    const int max_steps = cap > INT_MAX ? INT_MAX : static_cast<int>(cap);
    bool exhausted = false;
    for (;;) {
        if (L.state == ST_DONE) complete(s, a, ra, L, cold);
        const unsigned idle = __ballot_sync(FULL, L.state == ST_IDLE);
        if (!exhausted && idle != 0 && (__popc(idle) >= refill || idle == FULL)) {
            const int k = __popc(idle);
            const int leader = __ffs(idle) - 1;
            long long base = 0;
            if (lane == leader) base = atomicAdd(reinterpret_cast<unsigned long long *>(counter), static_cast<unsigned long long>(k));
            base = __shfl_sync(FULL, base, leader);
            if (base + k >= total) exhausted = true;
            if (L.state == ST_IDLE) {
                const long long item = base + __popc(idle & lanes_below);
                if (item < total) start_job(s, a, ra, L, cold, item, kinds, tiles_x, tiles_per_view);
            }
        }
        const unsigned busy = __ballot_sync(FULL, L.state != ST_IDLE);
        if (busy == 0) {
            if (exhausted) break;
            continue;
        }
        // Walk until enough lanes are free to be worth a refill (or, once the work is all taken, until all are).
        // Lanes at a leaf (an instance to enter, a triangle to test) wait while the others take internal-node
        // steps, and the warp takes a leaf step only once leaf_batch of them wait or no lane is at an internal
        // node: each kind of step then runs with many lanes instead of every kind running in every step. A
        // lane's own walk is unchanged, step for step.
        for (;;) {
            const bool walking = L.state == ST_WALK;
            const unsigned at_leaf = __ballot_sync(FULL, walking && L.count != 0);
            const unsigned at_inner = __ballot_sync(FULL, walking && L.count == 0);
            const unsigned busy_walk = at_leaf | at_inner;
            if (busy_walk == 0) break;
            if (!exhausted && 32 - __popc(busy_walk) >= refill) break;
            const bool leaf_phase = __popc(at_leaf) >= leaf_batch || at_inner == 0;
            if (walking && (L.count != 0) == leaf_phase) {
                if (++L.steps > max_steps) {  // a lane's own steps; only a malformed tree gets past the cap
                    *(kinds == KINDS_RAYS ? ra.error_flag : a.error_flag) = 2;
                    L.state = ST_DONE;
                } else if (leaf_phase) {
                    walk_leaf(s, L, cold, st, kinds == KINDS_RAYS ? ra.error_flag : a.error_flag);
                } else {
                    walk_inner(s, L, cold, st, kinds == KINDS_RAYS ? ra.error_flag : a.error_flag);
                }
            }
        }
    }
}

template <int THREADS, int MIN_BLOCKS>
cudaError_t launch_variant(const SceneParams &s, const RenderArgs &a, const RayArgs *rays, int *counter, int refill,
    int leaf_batch, cudaStream_t stream) {
    const int tiles_x = (a.width + 3) / 4, tiles_y = (a.rows + 3) / 4;
    const int tiles_per_view = tiles_x * tiles_y;
    const int kinds = rays ? KINDS_RAYS : (a.rgb ? 1 : 0) | ((a.depth || a.normal || a.object_id || a.hit_instance) ? 2 : 0);
    if (kinds == 0) return cudaSuccess;
    const long long total = rays ? rays->count : 16LL * tiles_per_view * a.views * (kinds == 3 ? 2 : 1);
    if (total == 0) return cudaSuccess;
    const RayArgs ra = rays ? *rays : RayArgs{};
    auto kernel = render_persistent_kernel<THREADS, MIN_BLOCKS>;
    const size_t smem = static_cast<size_t>(C_FIELDS) * THREADS * sizeof(float);
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    // Enough resident warps to fill every SM, and no more warps than there are jobs for.
    long long blocks = static_cast<long long>(sms) * per_sm;
    const long long needed = (total + THREADS - 1) / THREADS;
    if (blocks > needed) blocks = needed;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    if (!rays) {
        if (!a.basis_given) e = launch_prepare_cameras(a.cameras, a.views, a.camera_basis, stream);
        if (e != cudaSuccess) return e;
    }
    kernel<<<static_cast<unsigned>(blocks), THREADS, smem, stream>>>(s, a, ra, counter, total, kinds, tiles_x,
        tiles_per_view, refill, leaf_batch);
    return cudaGetLastError();
}

}  // namespace

// (threads per CTA, register budget) -> the instantiation with that budget; rays: a launch of ray queries.
cudaError_t launch_persistent(const SceneParams &s, const RenderArgs &a, const RayArgs *rays, int *counter,
    const PersistentTuning &t, cudaStream_t stream) {
    if (t.threads == 128 && t.registers == 64) return launch_variant<128, 8>(s, a, rays, counter, t.refill, t.leaf_batch, stream);
    if (t.threads == 128 && t.registers == 72) return launch_variant<128, 7>(s, a, rays, counter, t.refill, t.leaf_batch, stream);
    if (t.threads == 128 && t.registers == 48) return launch_variant<128, 10>(s, a, rays, counter, t.refill, t.leaf_batch, stream);
    if (t.threads == 256 && t.registers == 64) return launch_variant<256, 4>(s, a, rays, counter, t.refill, t.leaf_batch, stream);
    if (t.threads == 256 && t.registers == 48) return launch_variant<256, 5>(s, a, rays, counter, t.refill, t.leaf_batch, stream);
    if (t.threads == 64 && t.registers == 64) return launch_variant<64, 16>(s, a, rays, counter, t.refill, t.leaf_batch, stream);
    return cudaErrorInvalidValue;
}

cudaError_t launch_render_persistent(const SceneParams &s, const RenderArgs &a, int *counter, const PersistentTuning &t,
    cudaStream_t stream) {
    return launch_persistent(s, a, nullptr, counter, t, stream);
}

cudaError_t launch_rays_persistent(const SceneParams &s, const RayArgs &r, int *counter, const PersistentTuning &t,
    cudaStream_t stream) {
    return launch_persistent(s, RenderArgs{}, &r, counter, t, stream);
}

}  // namespace ngb
