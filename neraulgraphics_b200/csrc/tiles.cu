// The tile render kernels: the batched path's common case (one sample per pixel, at most one light, no mirror
// bounces), in three launches (camera rays, shading, shadow rays), for worlds of any size: candidate lists for
// worlds of up to TILE_MAX_INSTANCES instances (what a batch of simulator worlds holds), a packet walk of the
// world tree above that.
//
// One warp renders an 8 x 4 pixel tile of one view (the camera kernel, when a render asks for the picture and
// the centre-ray outputs: a 4 x 4 tile with a pixel's two rays on adjacent lanes, so its
// two nearly equal walks run side by side). All 32 rays of a tile start at the same eye and point into
// the same narrow pyramid, so in a world of up to TILE_MAX_INSTANCES instances the warp replaces the world
// tree's walk by one conservative test per instance, 32 instances at a time:
//   - lane j tests instance j's world box against the tile's pyramid (four planes through the eye, widened by
//     a margin far above rounding) and against the eye's distance; the ballot is the tile's candidate list,
//     sorted by the distance below which no ray of the tile can enter the box;
//   - every lane then visits the candidates in that order, the same instance at the same time across the warp,
//     so the mesh walks of neighbouring rays run together over the same nodes; a lane enters a candidate only
//     if its own ray passes the slab test of the instance's box (the test the world tree applies to that leaf),
//     with its closest hit so far as the limit, exactly as the world tree's walk does;
//   - the shadow rays of the tile go from the lit points to the light's sphere; the candidates for them are
//     the instances whose boxes meet the convex hull of those segments, tested on the coordinate axes and on
//     four axes tilted towards the light (separating axes of the hull).
// Why the hits are the reference's: a ray's slab test on a box inside a parent box never passes where the
// parent's fails (the subtraction, the product and min/max are monotone in correctly rounded arithmetic), so
// the world tree reaches an instance's leaf exactly when the ray passes the leaf's own box test; the walk
// inside a mesh is the reference's, order and all (src/mesh_dev.h:113-159). What can change is only the order
// in which instances are visited, and with it which of two hits within rounding of each other is kept, the
// near-ties the parity tests name. A shadow ray's any-hit answer does not depend on the order at all.
#include <climits>

#include "kernels.h"
#include "trace_common.cuh"

namespace ngb {
namespace {

using namespace tr;

constexpr unsigned FULL = 0xffffffffu;
constexpr int TILE_W = 8, TILE_H = 4;
constexpr int WALK_STACK = 64;      // a mesh's tree is at most 60 deep

// A tile's candidate instances as its warp holds them: each one's position in its world's run of sorted
// leaves and the distance below which no camera ray of the tile can enter its box, in the view's order of those
// distances (view_order_kernel). CAP: the most instances a world holds (32 or TILE_MAX_INSTANCES).
template <int CAP>
struct WarpSmem {
    int leaf[CAP];           // the candidates' leaves, smallest entry bound first (the view's order)
    float bound[CAP];        // and their bounds
};
// CAP 0: worlds of any size, walked as a packet (packet_walk); the warp's stack of the world tree's nodes.
template <>
struct WarpSmem<0> {
    int ref[TLAS_STACK];
    int count[TLAS_STACK];
};

__device__ __forceinline__ float warp_max(float v) { return from_ordered(__reduce_max_sync(FULL, to_ordered(v))); }
__device__ __forceinline__ float warp_min(float v) { return from_ordered(__reduce_min_sync(FULL, to_ordered(v))); }
__device__ __forceinline__ float abs_dot(float3 n, float3 h) { return fabsf(n.x) * h.x + fabsf(n.y) * h.y + fabsf(n.z) * h.z; }

// A world's run of sorted leaves: leaf k of world w is node n - 1 + first + k.
__device__ __forceinline__ const float4 *world_leaves(const SceneParams &s, int world) {
    return s.tlas + 2 * (static_cast<long long>(s.tlas_internal) + world_first_of(s, world));
}

// An instance's leaf as the world tree's walk handles it once the ray has passed the leaf's box: the ray
// moved to mesh space and the mesh root's box test (blas_walk, src/mesh_dev.h:164-175), then the mesh's tree
// from its child-pair records: the nearer child first (dl <= dr), the farther one pushed with its entry
// distance and dropped at pop time once a hit is closer (traverse, src/mesh_dev.h:113-159), and a leaf's
// triangles in order (mesh_intersect / mesh_occluded, src/mesh_dev.h:180-226).
// ANY (shadow rays): true at the first hit closer than tmax; tmax never shrinks, so a pushed node is never
// dropped at pop time and its entry distance is not checked. Otherwise: lowers tmax to each closer hit and
// records it, true if there was one. Inlined: every kernel calls it from one place (a call per visit costs the
// caller's registers saved and restored around it: camera 3.81 -> 3.55 ms at 4096 worlds).
template <bool ANY>
__device__ __forceinline__ bool instance_walk_body(const float4 *__restrict__ inst, const float *__restrict__ slot_bounds,
    const int2 *__restrict__ slot_root, const float4 *__restrict__ pairs, const float4 *__restrict__ tris,
    const float4 *__restrict__ slot_sphere, int id, float3 o, float3 d, float &tmax, int &hit_tri, float &hu,
    float &hv, int max_steps, int *err) {
    const float4 *rec = inst + 4 * static_cast<long long>(id);
    InstanceRec r;
    r.r0 = __ldg(rec);
    r.r1 = __ldg(rec + 1);
    r.r2 = __ldg(rec + 2);
    const int slot = __float_as_int(__ldg(rec + 3).y);
    o = to_local_point(r, o);
    d = to_local_dir(r, d);
    // A ray that passes farther from the mesh's sphere centre than its radius meets none of its triangles: the
    // squared distance |m x d|^2 / |d|^2 (m from the centre to the origin), against r^2 with a margin of 1e-3
    // relative plus 1e-4 |m|^2, far above the float rounding of the products.
    const float4 sph = __ldg(slot_sphere + slot);
    if (sph.w > 0.0f) {
        const float3 m = o - mk3(sph.x, sph.y, sph.z);
        const float dd = dot(d, d), b = dot(m, d), mm = dot(m, m);
        if (mm * dd - b * b > (sph.w * sph.w * 1.001f + 1e-4f * mm) * dd) return false;
    }
    const float3 inv = safe_inverse(d);
    const float *b = slot_bounds + 6 * slot;
    const float4 blo = make_float4(__ldg(b), __ldg(b + 1), __ldg(b + 2), 0.0f);
    const float4 bhi = make_float4(__ldg(b + 3), __ldg(b + 4), __ldg(b + 5), 0.0f);
    if (box_entry(blo, bhi, o, inv, tmax) >= NO_HIT) return false;
    const int2 root = __ldg(slot_root + slot);
    int ref = root.x, count = root.y;
    // One 16-byte entry per pushed node: (reference, count, entry distance), stored and loaded whole.
    int4 st[WALK_STACK];
    bool found = false;
    int sp = 0, steps = 0;
    // While-while: a lane walks internal nodes until it stands at a leaf (or its walk ends), and the leaf's
    // triangles are tested once the warp's lanes have all come out of the inner loop, so the two kinds of
    // step run with their own lanes together instead of every iteration paying for both.
    for (;;) {
        while (count == 0) {
            if (++steps > max_steps) {  // a correct walk visits each node once; only a malformed tree gets here
                *err = 2;
                return found;
            }
            const float4 *q = pairs + 4 * static_cast<long long>(ref);
            const float4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
            const float dl = box_entry(make_float4(q0.x, q0.y, q0.z, 0.0f), make_float4(q0.w, q1.x, q1.y, 0.0f), o, inv,
                tmax);
            const float dr = box_entry(make_float4(q1.z, q1.w, q2.x, 0.0f), make_float4(q2.y, q2.z, q2.w, 0.0f), o, inv,
                tmax);
            if (dl < NO_HIT || dr < NO_HIT) {
                const bool left_first = dl <= dr;
                const float far_t = left_first ? dr : dl;
                if (far_t < NO_HIT) {
                    if (sp >= WALK_STACK) {
                        *err = 1;
                        return found;
                    }
                    st[sp] = make_int4(__float_as_int(left_first ? q3.z : q3.x), __float_as_int(left_first ? q3.w : q3.y),
                        __float_as_int(far_t), 0);
                    ++sp;
                }
                ref = __float_as_int(left_first ? q3.x : q3.z);
                count = __float_as_int(left_first ? q3.y : q3.w);
            } else {
                int4 e = make_int4(0, 0, 0, 0);
                if (ANY) {
                    if (sp == 0) return false;
                    e = st[--sp];
                } else {
                    while (sp > 0) {
                        e = st[sp - 1];
                        if (__int_as_float(e.z) < tmax) break;
                        --sp;
                    }
                    if (sp == 0) return found;
                    --sp;
                }
                ref = e.x;
                count = e.y;
            }
        }
        if (++steps > max_steps) {
            *err = 2;
            return found;
        }
        for (int j = ref; j < ref + count; ++j) {
            float t, bu, bv;
            if (triangle_hit(tris, j, o, d, tmax, t, bu, bv)) {
                if (ANY) return true;
                tmax = t;
                hit_tri = j;
                hu = bu;
                hv = bv;
                found = true;
            }
        }
        int4 e = make_int4(0, 0, 0, 0);
        if (ANY) {
            if (sp == 0) return false;
            e = st[--sp];
        } else {
            while (sp > 0) {
                e = st[sp - 1];
                if (__int_as_float(e.z) < tmax) break;
                --sp;
            }
            if (sp == 0) return found;
            --sp;
        }
        ref = e.x;
        count = e.y;
    }
}

// A camera ray's closest mesh hit over the tile's candidates, visited by the whole warp in the same order.
// The warp stops once no lane's closest hit lies beyond the next candidate's entry bound.
template <int CAP>
__device__ __forceinline__ void closest_meshes(const SceneParams &s, const WarpSmem<CAP> &sm, const float4 *leaves,
    int ncand, bool active, float3 o, float3 d, float &tmax, int &hit_inst, int &hit_tri, float &hu, float &hv,
    int max_steps, int *err) {
    const float3 inv = safe_inverse(d);
    for (int c = 0; c < ncand; ++c) {
        const bool reach = active && sm.bound[c] < tmax;
        if (!__any_sync(FULL, reach)) break;
        const float4 *leaf = leaves + 2 * sm.leaf[c];
        const float4 lo = __ldg(leaf), hi = __ldg(leaf + 1);
        if (reach && box_entry(lo, hi, o, inv, tmax) < NO_HIT) {
            const int id = ~__float_as_int(lo.w);
            if (instance_walk_body<false>(s.inst, s.slot_bounds, s.slot_root, s.blas_pairs, s.tris, s.slot_sphere, id, o, d,
                    tmax, hit_tri, hu, hv, max_steps, err))
                hit_inst = id;
        }
    }
}

// A world's tree walked by the whole warp together (a packet), for the camera rays of worlds too large for
// candidate lists: every internal node that some lane's ray enters before its closest hit so far is visited
// once for all lanes, from child-pair records, the child the lanes enter first (least entry distance over the
// lanes) before the other; an instance whose box a lane's ray enters is walked by that lane (instance_walk_body).
// Each lane gets the hit its own walk of the tree finds, up to which of two equally distant hits is kept (the
// instance order differs from a single ray's). The stack lives in the warp's shared memory.
// ANY (shadow rays): a lane stops at its first hit closer than tmax (hit_inst set to that instance), and the
// packet ends once every lane has stopped; the answer does not depend on the order. skip: an instance the lane
// leaves out (-1: none).
template <bool ANY>
__device__ __forceinline__ void packet_walk(const SceneParams &s, WarpSmem<0> &sm, int lane, int world, bool active,
    float3 o, float3 d, float &tmax, int &hit_inst, int &hit_tri, float &hu, float &hv, int skip, int max_steps,
    int *err) {
    const int root = s.instance_count > 0 ? __ldg(s.roots + world) : -1;
    if (root < 0) return;
    const float3 inv = safe_inverse(d);
    int ref = root, count = 0, sp = 0;
    if (root >= s.tlas_internal) {  // a world of one instance: its leaf is the root, taken as an instance met on the stack
        ref = ~__float_as_int(__ldg(s.tlas + 2 * root).w);
        count = -1;
    } else {
        const float4 lo = __ldg(s.tlas + 2 * root), hi = __ldg(s.tlas + 2 * root + 1);
        if (!__any_sync(FULL, active && box_entry(lo, hi, o, inv, tmax) < NO_HIT)) return;
    }
    const int max_nodes = 2 * s.instance_count + 2;
    for (int steps = 0;; ++steps) {
        if (steps > max_nodes) {  // a correct walk visits each node once; only a malformed tree gets here
            if (lane == 0) *err = 2;
            return;
        }
        if (ANY && !__any_sync(FULL, active)) return;
        bool pop = true;
        // The instance this step meets, if any, and whether the lane's ray enters its leaf box: walked by that
        // lane, at one place below (so the walk is inlined).
        int meet = -1;
        bool enters = false;
        if (count < 0) {
            // An instance met on the stack: its leaf box first (leaf k of the sorted leaves is node n - 1 + k).
            const float4 *leaf = s.tlas + 2 * (static_cast<long long>(s.tlas_internal) + __ldg(s.leaf_of + ref));
            meet = ref;
            enters = active && box_entry(__ldg(leaf), __ldg(leaf + 1), o, inv, tmax) < NO_HIT;
        } else {
            const float4 *q = s.tlas_pairs + 4 * static_cast<long long>(ref);
            const float4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
            const bool open = active;
            const float dl = open ? box_entry(make_float4(q0.x, q0.y, q0.z, 0.0f), make_float4(q0.w, q1.x, q1.y, 0.0f), o,
                inv, tmax) : NO_HIT;
            const float dr = open ? box_entry(make_float4(q1.z, q1.w, q2.x, 0.0f), make_float4(q2.y, q2.z, q2.w, 0.0f), o,
                inv, tmax) : NO_HIT;
            const bool hl = __any_sync(FULL, dl < NO_HIT), hr = __any_sync(FULL, dr < NO_HIT);
            if (hl || hr) {
                const bool left_first = !hr || (hl && warp_min(dl) <= warp_min(dr));
                const int near_ref = __float_as_int(left_first ? q3.x : q3.z);
                const int near_count = __float_as_int(left_first ? q3.y : q3.w);
                if (hl && hr) {
                    if (sp >= TLAS_STACK) {
                        if (lane == 0) *err = 1;
                        return;
                    }
                    if (lane == 0) {
                        sm.ref[sp] = __float_as_int(left_first ? q3.z : q3.x);
                        sm.count[sp] = __float_as_int(left_first ? q3.w : q3.y);
                    }
                    ++sp;
                }
                if (near_count < 0) {
                    meet = near_ref;
                    enters = (left_first ? dl : dr) < NO_HIT;
                } else {
                    ref = near_ref;
                    count = near_count;
                    pop = false;
                }
            }
        }
        if (ANY) {
            float tm = tmax;
            if (enters && meet != skip && instance_walk_body<true>(s.inst, s.slot_bounds, s.slot_root, s.blas_pairs,
                                              s.tris, s.slot_sphere, meet, o, d, tm, hit_tri, hu, hv, max_steps, err)) {
                hit_inst = meet;
                active = false;
            }
        } else if (enters && instance_walk_body<false>(s.inst, s.slot_bounds, s.slot_root, s.blas_pairs, s.tris,
                                 s.slot_sphere, meet, o, d, tmax, hit_tri, hu, hv, max_steps, err)) {
            hit_inst = meet;
        }
        if (pop) {
            __syncwarp();
            if (sp == 0) return;
            --sp;
            ref = sm.ref[sp];
            count = sm.count[sp];
            __syncwarp();
        }
    }
}

// Spheres and the floor before the meshes, the meshes with the closest of those as their limit
// (scene_intersect, src/render_core.h:78-112).
__device__ __forceinline__ float spheres_and_floor(const SceneParams &s, float3 o, float3 d, int &best_sphere,
    bool &hit_floor) {
    float best = 1e30f;
    best_sphere = -1;
    for (int i = 0; i < s.sphere_count; ++i) {
        float t;
        if (sphere_hit(s.spheres[i], o, d, t) && t < best) {
            best = t;
            best_sphere = i;
        }
    }
    hit_floor = false;
    float dd;
    if (floor_hit(s.floor, o, d, best, dd)) {
        best = dd;
        hit_floor = true;
    }
    return best;
}

// The surface of a closest hit, as scene_intersect resolves it (src/render_core.h:116-141).
__device__ __forceinline__ void resolve(const SceneParams &s, int world, float3 point, float3 d, int hit_inst,
    int hit_tri, float hu, float hv, int best_sphere, bool hit_floor, float3 &normal, DevMaterial &mat, int &object) {
    if (hit_inst >= 0) {
        normal = mesh_surface(s, hit_inst, hit_tri, hu, hv, d);
        mat = s.slot_material[table_of(s, hit_inst, world)];
        object = OBJECT_INSTANCE + (hit_inst - world_first_of(s, world));
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

// sample_pixel's average of one sample, sRGB, bytes (src/render_core.h:248-283), packed r | g << 8 | b << 16.
// Inlined at both of the shade kernel's uses (0.62 -> 0.61 ms at 4096 worlds against one shared copy).
__device__ __forceinline__ int rgb_bytes(const float *table, float3 radiance) { return rgb_packed(table, radiance); }

__device__ __forceinline__ void put_rgb(uint8_t *rgb, long long pix, int bytes) {
    uint8_t *o = rgb + 3 * static_cast<size_t>(pix);
    o[0] = static_cast<uint8_t>(bytes);
    o[1] = static_cast<uint8_t>(bytes >> 8);
    o[2] = static_cast<uint8_t>(bytes >> 16);
}


// i / per and i % per (per > 0), in 32 bits whenever i fits: a 64-bit division is a long instruction
// sequence, paid once per tile by every kernel that walks tiles.
__device__ __forceinline__ int split_index(long long i, int per, int &rem) {
    if (i <= 0xffffffffLL) {
        const unsigned u = static_cast<unsigned>(i), p = static_cast<unsigned>(per);
        const unsigned q = u / p;
        rem = static_cast<int>(u - q * p);
        return static_cast<int>(q);
    }
    rem = static_cast<int>(i % per);
    return static_cast<int>(i / per);
}

// The tile kernels' common start: which tile of which view, and the pixel of this lane.
struct TileAt {
    int view, world, x0, y0, x, y;
    int width, height;  // the view's image
    float aspect;
    bool pixel;
    long long pix;
};

__device__ __forceinline__ TileAt tile_at(const RenderArgs &a, long long tile, int tiles_x, int tiles_per_view, int lane) {
    TileAt t;
    int q, row0, row_end;  // the view's rendered rows [row0, row_end)
    long long first_pixel;
    if (a.view_info) {
        t.view = view_of(a.view_info, a.views, tile, true);
        const int4 v = __ldg(a.view_info + t.view);
        t.width = v.x;
        t.height = v.y;
        t.aspect = static_cast<float>(v.x) / static_cast<float>(v.y);
        tiles_x = (v.x + TILE_W - 1) / TILE_W;
        q = static_cast<int>(tile - v.w);
        first_pixel = v.z;
        row0 = 0;
        row_end = v.y;
    } else {
        t.view = split_index(tile, tiles_per_view, q);
        t.width = a.width;
        t.height = a.height;
        t.aspect = a.aspect;
        first_pixel = static_cast<long long>(t.view) * a.rows * a.width;
        row0 = a.row_first;
        row_end = a.row_first + a.rows;
    }
    t.x0 = (q % tiles_x) * TILE_W;
    t.y0 = row0 + (q / tiles_x) * TILE_H;
    t.x = t.x0 + (lane % TILE_W);
    t.y = t.y0 + lane / TILE_W;
    t.pixel = t.x < t.width && t.y < row_end;
    t.world = t.view / a.cameras_per_world;
    t.pix = first_pixel + static_cast<long long>(t.y - row0) * t.width + t.x;
    return t;
}

// The camera kernel's tiles when a render asks for the picture and the centre-ray outputs: 4 x 4 pixels, lanes 2k and 2k + 1 on pixel k (k = 0..15, row-major), the even lane tracing the centre
// ray and the odd one the picture ray, so the two nearly equal walks of a pixel run side by side.
__device__ __forceinline__ TileAt pair_tile_at(const RenderArgs &a, long long tile, int tiles_x, int tiles_per_view,
    int lane) {
    TileAt t;
    int q, row0, row_end;  // the view's rendered rows [row0, row_end)
    long long first_pixel;
    if (a.view_info) {
        // Uneven views: the last view whose first 4 x 4 tile is at most tile.
        int lo = 0, hi = a.views - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(a.view_pair_tile + mid) <= tile) lo = mid;
            else hi = mid - 1;
        }
        t.view = lo;
        const int4 v = __ldg(a.view_info + lo);
        t.width = v.x;
        t.height = v.y;
        t.aspect = static_cast<float>(v.x) / static_cast<float>(v.y);
        tiles_x = (v.x + 3) / 4;
        q = static_cast<int>(tile - __ldg(a.view_pair_tile + lo));
        first_pixel = v.z;
        row0 = 0;
        row_end = v.y;
    } else {
        t.view = split_index(tile, tiles_per_view, q);
        t.width = a.width;
        t.height = a.height;
        t.aspect = a.aspect;
        first_pixel = static_cast<long long>(t.view) * a.rows * a.width;
        row0 = a.row_first;
        row_end = a.row_first + a.rows;
    }
    const int k = lane >> 1;
    t.x0 = (q % tiles_x) * 4;
    t.y0 = row0 + (q / tiles_x) * 4;
    t.x = t.x0 + (k & 3);
    t.y = t.y0 + (k >> 2);
    t.pixel = t.x < t.width && t.y < row_end;
    t.world = t.view / a.cameras_per_world;
    t.pix = first_pixel + static_cast<long long>(t.y - row0) * t.width + t.x;
    return t;
}

// One CTA per view: its world's instances in the order the view's tiles walk their candidates, nearest bound first
// (the eye's distance to the instance's leaf box, 1e-5 under it: no camera ray of the view can enter the box
// closer), ties by leaf order. The bound depends on the eye alone, so every tile of the view takes this order and
// keeps only its own candidates.
template <int CAP>
__global__ void __launch_bounds__(128) view_order_kernel(const __grid_constant__ SceneParams s, const RenderArgs a) {
    __shared__ float bound[CAP];
    const int view = blockIdx.x;
    const int world = view / a.cameras_per_world;
    const int P = s.instance_count > 0 ? world_count_of(s, world) : 0;
    const float4 c0 = __ldg(a.camera_basis + 3 * view);
    const float3 eye = mk3(c0.x, c0.y, c0.z);
    const float4 *leaves = world_leaves(s, world);
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        const float4 lo = __ldg(leaves + 2 * j), hi = __ldg(leaves + 2 * j + 1);
        const float dx = fmaxf(fmaxf(lo.x - eye.x, eye.x - hi.x), 0.0f);
        const float dy = fmaxf(fmaxf(lo.y - eye.y, eye.y - hi.y), 0.0f);
        const float dz = fmaxf(fmaxf(lo.z - eye.z, eye.z - hi.z), 0.0f);
        bound[j] = sqrtf(dx * dx + dy * dy + dz * dz) * 0.99999f;
    }
    __syncthreads();
    int *order = a.view_order + static_cast<long long>(view) * a.order_stride;
    float *order_bound = a.view_bound + static_cast<long long>(view) * a.order_stride;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const float bi = bound[i];
        int rank = 0;
        for (int k = 0; k < P; ++k) {
            const float bk = bound[k];
            rank += (bk < bi) || (bk == bi && k < i);
        }
        order[rank] = i;
        order_bound[rank] = bi;
    }
}

// A warp's next run of tiles, fetch of them from one atomic (32 rays each; a tuning choice: 1 gives the finest
// balance at the end of a launch, more fewer atomics); first >= tiles when none are left.
__device__ __forceinline__ long long fetch_tiles(int *counter, int lane, int fetch) {
    long long first = 0;
    if (lane == 0)
        first = static_cast<long long>(atomicAdd(reinterpret_cast<unsigned long long *>(counter),
            static_cast<unsigned long long>(fetch)));
    return __shfl_sync(FULL, first, 0);
}

// The picture ray of pixel (x, y): its jitter draws from the pixel's random stream, which is left where the
// light sample continues it (sample_pixel, src/render_core.h:248-258).
__device__ __forceinline__ float3 picture_ray(const RenderArgs &a, int x, int y, int width, int height, float aspect,
    float3 right, float3 up, float3 fwd, uint32_t &rng) {
    rng = pcg_hash(static_cast<uint32_t>(y * width + x) ^ pcg_hash(static_cast<uint32_t>(a.frame) + 1u));
    const float jx = rand_float(rng);
    const float jy = rand_float(rng);
    return camera_dir(right, up, fwd, static_cast<float>(x) + jx, static_cast<float>(y) + jy, static_cast<float>(width),
        static_cast<float>(height), a.fov_scale, aspect);
}

// The picture ray's closest hit as the camera kernel hands it to the shade kernel: the object code
// (instance >= 0, else -1 nothing, -2 the floor, -3 - i sphere i).
constexpr int CODE_NONE = -1, CODE_FLOOR = -2, CODE_SPHERE = -3;

// Camera kernel. THREADS per CTA and MIN_BLOCKS resident CTAs per SM set the register budget. Per tile: the
// candidates, then the centre rays (depth, normals, IDs written here) and the picture rays (their closest
// hits written for the shade kernel).
template <int THREADS, int MIN_BLOCKS, int CAP, bool PAIRED>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) camera_tiles_kernel(const __grid_constant__ SceneParams s,
    const RenderArgs a, int *counter, long long tiles, int tiles_x, int tiles_per_view, int fetch) {
    __shared__ WarpSmem<CAP> warp_smem[THREADS / 32];
    WarpSmem<CAP> &sm = warp_smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int max_steps = s.blas_node_count + 2;
    const bool want_aov = a.depth || a.normal || a.object_id || a.hit_instance;
    const float fs = a.fov_scale;
    for (;;) {
        const long long first = fetch_tiles(counter, lane, fetch);
        if (first >= tiles) break;
        const long long last = first + fetch < tiles ? first + fetch : tiles;
        for (long long tile = first; tile < last; ++tile) {
            const TileAt T = PAIRED ? pair_tile_at(a, tile, tiles_x, tiles_per_view, lane)
                                    : tile_at(a, tile, tiles_x, tiles_per_view, lane);
            constexpr int TW = PAIRED ? 4 : TILE_W, TH = PAIRED ? 4 : TILE_H;
            const int P = s.instance_count > 0 ? world_count_of(s, T.world) : 0;
            const float fw = static_cast<float>(T.width), fh = static_cast<float>(T.height), asp = T.aspect;
            // The view's camera (camera_from_matrix, src/render_core.h:264-273).
            const float4 c0 = __ldg(a.camera_basis + 3 * T.view), c1 = __ldg(a.camera_basis + 3 * T.view + 1);
            const float4 c2 = __ldg(a.camera_basis + 3 * T.view + 2);
            const float3 eye = mk3(c0.x, c0.y, c0.z), right = mk3(c0.w, c1.x, c1.y);
            const float3 up = mk3(c1.z, c1.w, c2.x), fwd = mk3(c2.y, c2.z, c2.w);

            const float4 *leaves = world_leaves(s, T.world);
            int ncand = 0;
            if constexpr (CAP > 0) {
            // The tile's pyramid: the tangent-plane offsets of its pixel edges (every jittered and centre ray of
            // the tile lies inside), widened by 1e-3, and the four side planes through the eye, facing inwards.
            // The offsets need no exact division: their rounding (a few ulp from the fast reciprocal) lies far
            // inside the widening.
            const float rw = __fdividef(2.0f, fw), rh = __fdividef(2.0f, fh);
            const float sxa = (static_cast<float>(T.x0) * rw - 1.0f) * fs * asp;
            const float sxb = (static_cast<float>(T.x0 + TW) * rw - 1.0f) * fs * asp;
            const float sya = -(static_cast<float>(T.y0) * rh - 1.0f) * fs;
            const float syb = -(static_cast<float>(T.y0 + TH) * rh - 1.0f) * fs;
            const float sx_lo = fminf(sxa, sxb) - 1e-3f * (1.0f + fabsf(sxa) + fabsf(sxb));
            const float sx_hi = fmaxf(sxa, sxb) + 1e-3f * (1.0f + fabsf(sxa) + fabsf(sxb));
            const float sy_lo = fminf(sya, syb) - 1e-3f * (1.0f + fabsf(sya) + fabsf(syb));
            const float sy_hi = fmaxf(sya, syb) + 1e-3f * (1.0f + fabsf(sya) + fabsf(syb));

            // Every instance of the world against the pyramid, 32 at a time, in the view's order (nearest bound
            // first, ties by leaf order): the candidates, already in the order they are walked.
            const float3 k00 = right * sx_lo + up * sy_lo + fwd, k10 = right * sx_hi + up * sy_lo + fwd;
            const float3 k11 = right * sx_hi + up * sy_hi + fwd, k01 = right * sx_lo + up * sy_hi + fwd;
            const float3 mid = k00 + k11;
            float3 planes[4] = {cross(k00, k10), cross(k10, k11), cross(k11, k01), cross(k01, k00)};
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (dot(planes[e], mid) < 0.0f) planes[e] = -planes[e];
            const int *order = a.view_order + static_cast<long long>(T.view) * a.order_stride;
            const float *order_bound = a.view_bound + static_cast<long long>(T.view) * a.order_stride;
            __syncwarp();
            for (int base = 0; base < P; base += 32) {
                const int k = base + lane;
                bool cand = false;
                int j = 0;
                float bound = 0.0f;
                if (k < P) {
                    j = __ldg(order + k);
                    bound = __ldg(order_bound + k);
                    const float4 lo = __ldg(leaves + 2 * j), hi = __ldg(leaves + 2 * j + 1);
                    const float3 c = mk3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
                    const float3 h = mk3(0.5f * (hi.x - lo.x), 0.5f * (hi.y - lo.y), 0.5f * (hi.z - lo.z));
                    const float3 rel = c - eye;
                    const float pad = 1e-4f * (fabsf(rel.x) + fabsf(rel.y) + fabsf(rel.z) + h.x + h.y + h.z) + 1e-4f;
                    cand = true;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float3 n = planes[e];
                        const float reach = dot(n, rel) + abs_dot(n, h) + pad * (fabsf(n.x) + fabsf(n.y) + fabsf(n.z));
                        if (reach < 0.0f) cand = false;
                    }
                }
                const unsigned cmask = __ballot_sync(FULL, cand);
                if (cand) {
                    const int at = ncand + __popc(cmask & below);
                    sm.leaf[at] = j;
                    sm.bound[at] = bound;
                }
                ncand += __popc(cmask);
            }
            __syncwarp();
            }

            // The centre ray for depth, normals and IDs (aov_pixel, src/render_core.h:313-327), then the picture
            // ray (trace, src/render_core.h:202-245) up to its closest hit. Spheres and the floor first.
            // Paired tiles: one pass, each lane its own kind of ray (the trip count is the same on every lane).
            const int first_pass = PAIRED ? (lane & 1) : (want_aov ? 0 : 1);
            const int last_pass = PAIRED ? (lane & 1) : (a.rgb ? 1 : 0);
            for (int pass = first_pass; pass <= last_pass; ++pass) {
                float3 d;
                if (pass == 0) {
                    d = camera_dir(right, up, fwd, static_cast<float>(T.x) + 0.5f, static_cast<float>(T.y) + 0.5f, fw, fh,
                        fs, asp);
                } else {
                    uint32_t rng;
                    d = picture_ray(a, T.x, T.y, T.width, T.height, asp, right, up, fwd, rng);
                }
                int best_sphere;
                bool hit_floor;
                float tmax = spheres_and_floor(s, eye, d, best_sphere, hit_floor);
                int hit_inst = -1, hit_tri = -1;
                float hu = 0.0f, hv = 0.0f;
                if constexpr (CAP > 0) {
                    closest_meshes(s, sm, leaves, ncand, T.pixel, eye, d, tmax, hit_inst, hit_tri, hu, hv, max_steps,
                        a.error_flag);
                } else {
                    packet_walk<false>(s, sm, lane, T.world, T.pixel, eye, d, tmax, hit_inst, hit_tri, hu, hv, -1,
                        max_steps, a.error_flag);
                }
                if (!T.pixel) continue;
                const size_t p = static_cast<size_t>(T.pix);
                if (pass == 1) {
                    a.pic_hit[p] = make_float4(tmax, hu, hv, __int_as_float(hit_tri));
                    a.pic_code[p] = hit_inst >= 0 ? hit_inst
                        : hit_floor           ? CODE_FLOOR
                        : best_sphere >= 0    ? CODE_SPHERE - best_sphere
                                              : CODE_NONE;
                    continue;
                }
                const bool mesh = hit_inst >= 0;
                const bool found = mesh || best_sphere >= 0 || hit_floor;
                float3 normal = mk3(0.0f, 0.0f, 0.0f);
                DevMaterial mat{};
                int object = OBJECT_NONE;
                // The object ID needs only which object was hit; the surface (normal, material) only when normals
                // are asked for.
                if (found && a.normal) {
                    resolve(s, T.world, eye + d * tmax, d, hit_inst, hit_tri, hu, hv, best_sphere, hit_floor, normal,
                        mat, object);
                } else if (found) {
                    object = mesh ? OBJECT_INSTANCE + (hit_inst - world_first_of(s, T.world))
                        : hit_floor ? OBJECT_FLOOR
                                    : OBJECT_SPHERE + best_sphere;
                }
                if (a.depth) a.depth[p] = found ? tmax * dot(d, fwd) : __int_as_float(0x7f800000);
                if (a.normal) {
                    a.normal[3 * p] = normal.x;
                    a.normal[3 * p + 1] = normal.y;
                    a.normal[3 * p + 2] = normal.z;
                }
                if (a.object_id) a.object_id[p] = object;
                if (a.hit_instance) {
                    a.hit_instance[p] = mesh ? hit_inst : -1;
                    a.hit_triangle[p] = mesh ? __ldg(s.tri_index + hit_tri) : -1;
                    a.hit_u[p] = mesh ? hu : 0.0f;
                    a.hit_v[p] = mesh ? hv : 0.0f;
                }
            }
        }
    }
}

// Whether a shadow ray that leaves a mesh hit cannot meet that mesh again: the mesh is convex (host.h:
// mesh_hull), the hit face's normal facing the picture ray points away from the mesh's body, the shading normal
// agrees with it (so the ray starts 1e-3 * cos above the face's plane) and the ray moves away from that plane.
// The whole body lies below the plane, within 1e-6 of its radius, so no triangle of it can be met; the margin
// asked of the start (at least 1e-4 with the shading normal within 84 degrees of the face's) stays far above
// the rounding of the coordinates and of the convexity test.
__device__ __forceinline__ bool shadow_misses_own_mesh(const SceneParams &s, int world, int g, int tri, float hu,
    float hv, float3 dir, float3 shading, float3 light_dir, float3 point) {
    const float4 hull = __ldg(s.slot_hull + table_of(s, g, world));
    if (!(hull.w > 0.0f)) return false;
    const float4 *rec = s.inst + 4LL * g;
    const float3 r0 = xyz(__ldg(rec)), r1 = xyz(__ldg(rec + 1)), r2 = xyz(__ldg(rec + 2));
    const float3 v0 = xyz(__ldg(s.tris + 3LL * tri)), e1 = xyz(__ldg(s.tris + 3LL * tri + 1));
    const float3 e2 = xyz(__ldg(s.tris + 3LL * tri + 2));
    const float3 nl = cross(e1, e2);
    const float3 nw = r0 * nl.x + r1 * nl.y + r2 * nl.z;  // the face normal in the world (inverse-transpose)
    const float nw_len = sqrtf(dot(nw, nw)), nl_len = sqrtf(dot(nl, nl));
    float3 ng = nw * (1.0f / nw_len);
    float sigma = 1.0f;
    if (dot(ng, dir) > 0.0f) {
        ng = -ng;
        sigma = -1.0f;
    }
    const float3 pl = v0 + e1 * hu + e2 * hv;
    if (!(dot(mk3(hull.x, hull.y, hull.z) - pl, nl) * sigma < -5e-4f * hull.w * nl_len)) return false;
    const float cos_sg = dot(shading, ng);
    if (!(cos_sg > 0.1f) || !(dot(light_dir, ng) > 0.0f)) return false;
    // A vertex h above the face's plane in the mesh's frame (along the unit normal) lies h * |nl| / |nw| above it
    // in the world.
    const float above = 1e-6f * hull.w * nl_len / nw_len;
    const float mag = fmaxf(fmaxf(fabsf(point.x), fabsf(point.y)), fmaxf(fabsf(point.z), 1.0f));
    return 1e-3f * cos_sg > 2e-5f * mag + above;
}

// Shade kernel: one thread per pixel, straight-line code. The picture ray's hit resolved and lit (trace's
// first bounce, src/render_core.h:202-245): a pixel with nothing left to trace gets its bytes here; a lit
// surface leaves its shadow ray (origin, light distance) (direction, lit bytes) and its shadowed bytes (over
// the hit's code) for the shadow kernel. shadow_o.w = 0 marks a pixel without a shadow ray.
// RADIANCE: a single-view render's kernel (a.radiance set), keeping each pixel's radiance for its running average;
// otherwise the batch's, writing bytes.
template <bool RADIANCE>
__global__ void __launch_bounds__(256) shade_kernel(const __grid_constant__ SceneParams s, const RenderArgs a,
    long long pixels) {
    const long long per_view = static_cast<long long>(a.width) * a.rows;
    const float3 zero = mk3(0.0f, 0.0f, 0.0f);
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < pixels;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        int view, rem, row0 = 0, width = a.width, height = a.height;
        float aspect = a.aspect;
        if (a.view_info) {
            view = view_of(a.view_info, a.views, p, false);
            const int4 v = __ldg(a.view_info + view);
            width = v.x;
            height = v.y;
            aspect = static_cast<float>(v.x) / static_cast<float>(v.y);
            rem = static_cast<int>(p - v.z);
        } else {
            view = static_cast<int>(p / per_view);
            rem = static_cast<int>(p % per_view);
            row0 = a.row_first;
        }
        const int y = row0 + rem / width, x = rem % width;
        const int world = view / a.cameras_per_world;
        const float4 c0 = __ldg(a.camera_basis + 3 * view), c1 = __ldg(a.camera_basis + 3 * view + 1);
        const float4 c2 = __ldg(a.camera_basis + 3 * view + 2);
        const float3 eye = mk3(c0.x, c0.y, c0.z), right = mk3(c0.w, c1.x, c1.y);
        const float3 up = mk3(c1.z, c1.w, c2.x), fwd = mk3(c2.y, c2.z, c2.w);
        uint32_t rng;
        const float3 d = picture_ray(a, x, y, width, height, aspect, right, up, fwd, rng);
        const int code = a.pic_code[p];
        const float4 h = a.pic_hit[p];
        float3 radiance, shadowed = zero;
        float3 self_normal = zero, self_point = zero;  // the picture hit's shading normal and point
        bool pending = false;
        float3 so = zero, sd = zero;
        float sdist = 0.0f;
        int lit_bytes = 0, shadow_bytes = 0;
        if (code == CODE_NONE) {
            const float t = saturate(dot(d, s.env_up) * 0.5f + 0.5f);
            const float3 sky = (s.env_color_down + (s.env_color_up - s.env_color_down) * t) * s.env_intensity;
            radiance = zero + sky * 1.0f;
        } else {
            const float tmax = h.x;
            const int hit_inst = code >= 0 ? code : -1;
            const bool hit_floor = code == CODE_FLOOR;
            const int best_sphere = code <= CODE_SPHERE ? CODE_SPHERE - code : -1;
            const float3 point = eye + d * tmax;
            float3 normal;
            DevMaterial mat;
            int object;
            resolve(s, world, point, d, hit_inst, __float_as_int(h.w), h.y, h.z, best_sphere, hit_floor, normal, mat, object);
            self_normal = normal;
            self_point = point;
            radiance = radiance_of(mat, s.ambient, zero, zero);
            if (s.light_count == 1) {
                const DevLight &lt = s.lights[0];
                const float z = 1.0f - 2.0f * rand_float(rng);
                const float rad = sqrtf(fmaxf(0.0f, 1.0f - z * z));
                const float phi = 6.28318530718f * rand_float(rng);
                float sin_phi, cos_phi;
                sincosf(phi, &sin_phi, &cos_phi);
                const float3 lp = lt.position + mk3(rad * cos_phi, rad * sin_phi, z) * lt.radius;
                const float3 to_light = lp - point;
                const float light_distance = sqrtf(dot(to_light, to_light));
                const float3 light_dir = to_light * (1.0f / light_distance);
                const float strength = lt.intensity * light_factor(lt, light_dir, light_distance);
                if (strength > 0.0f) {
                    // The shadow ray: spheres and the floor here (scene_occluded, src/render_core.h:146-161).
                    so = offset_origin(point, normal, light_dir);
                    sd = light_dir;
                    sdist = light_distance;
                    bool blocked = false;
                    for (int i = 0; i < s.sphere_count && !blocked; ++i) {
                        float t;
                        if (sphere_hit(s.spheres[i], so, sd, t) && t < sdist) blocked = true;
                    }
                    if (!blocked) {
                        float dd;
                        blocked = floor_hit(s.floor, so, sd, sdist, dd);
                    }
                    if (!blocked) {
                        const float3 lit = lt.color * strength;
                        const float3 diffuse = zero + lit * fmaxf(0.0f, dot(light_dir, normal));
                        const float3 specular =
                            zero + lit * powf(fmaxf(0.0f, dot(reflect(light_dir, normal), d)), mat.exponent);
                        if (RADIANCE) shadowed = radiance;
                        else shadow_bytes = rgb_bytes(s.srgb_table, radiance);
                        radiance = radiance_of(mat, s.ambient, diffuse, specular);
                        pending = true;
                    }
                }
            }
        }
        int bytes = 0;
        if (RADIANCE) {
            // A single-view render keeps the sample's radiance (sample_pixel's sum over one sample) for its running
            // average: the lit one, which a blocking shadow ray replaces with the shadowed one (kept in pic_hit).
            const float3 lit = (zero + radiance) * (1.0f / 1.0f);
            a.radiance[p] = make_float4(lit.x, lit.y, lit.z, 0.0f);
        } else {
            bytes = rgb_bytes(s.srgb_table, radiance);
            // A shadow ray whose answer cannot change the pixel (lit and shadowed bytes equal, as where the surface
            // faces away from the light and the highlight rounds away) is not traced: the bytes are final here.
            if (pending && bytes == shadow_bytes) pending = false;
        }
        if (pending) {
            lit_bytes = bytes;
            // The shadow ray's own mesh: walked first when the ray starts on its body's side (the light is behind
            // the surface), left out when it cannot be met (shadow_misses_own_mesh), else walked in turn.
            int self = -1;
            if (code >= 0) {
                if (dot(sd, self_normal) < 0.0f) self = code * 4 + 2;
                else if (shadow_misses_own_mesh(s, world, code, __float_as_int(h.w), h.y, h.z, d, self_normal, sd,
                             self_point))
                    self = code * 4 + 1;
            }
            a.shadow_self[p] = self;
            a.shadow_o[p] = make_float4(so.x, so.y, so.z, sdist);
            a.shadow_d[p] = make_float4(sd.x, sd.y, sd.z, __int_as_float(lit_bytes));
            if (RADIANCE) {
                const float3 dark = (zero + shadowed) * (1.0f / 1.0f);
                a.pic_hit[p] = make_float4(dark.x, dark.y, dark.z, 0.0f);
            } else {
                a.pic_code[p] = shadow_bytes;
            }
        } else {
            if (!RADIANCE) put_rgb(a.rgb, p, bytes);
            a.shadow_o[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
}

// Shadow kernel: per tile, the shadow rays the shade kernel left. The candidates are the instances whose
// boxes meet the convex hull of the tile's segments from the shadow origins to their ends at the light.
// Separating axes: x, y and z, the direction away from the light, and four axes tilted from the sideways
// directions towards the light by the light sphere's angular radius, which hug the hull's sides. Each support
// is taken over the segments' own end points, so any axis is a valid test; these make it a tight one.
template <int THREADS, int MIN_BLOCKS, int CAP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) shadow_tiles_kernel(const __grid_constant__ SceneParams s,
    const RenderArgs a, int *counter, long long tiles, int tiles_x, int tiles_per_view, int fetch) {
    __shared__ int warp_cand[THREADS / 32][CAP];
    int *cand_leaf = warp_cand[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int max_steps = s.blas_node_count + 2;
    const DevLight &lt = s.lights[0];
    const float INF = __int_as_float(0x7f800000);
    for (;;) {
        const long long first = fetch_tiles(counter, lane, fetch);
        if (first >= tiles) break;
        const long long last = first + fetch < tiles ? first + fetch : tiles;
        for (long long tile = first; tile < last; ++tile) {
            const TileAt T = tile_at(a, tile, tiles_x, tiles_per_view, lane);
            const int P = s.instance_count > 0 ? world_count_of(s, T.world) : 0;
            float4 o4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (T.pixel) o4 = a.shadow_o[T.pix];
            const bool pending = o4.w > 0.0f;
            const unsigned shadow_lanes = __ballot_sync(FULL, pending);
            if (shadow_lanes == 0) continue;
            float4 d4 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
            if (pending) d4 = a.shadow_d[T.pix];
            const float3 so = mk3(o4.x, o4.y, o4.z), sd = mk3(d4.x, d4.y, d4.z);
            const float sdist = o4.w;
            int ncand = 0;
            const float4 *leaves = world_leaves(s, T.world);
            const float3 se = so + sd * sdist;
            const float mnx = warp_min(pending ? fminf(so.x, se.x) : INF);
            const float mny = warp_min(pending ? fminf(so.y, se.y) : INF);
            const float mnz = warp_min(pending ? fminf(so.z, se.z) : INF);
            const float mxx = warp_max(pending ? fmaxf(so.x, se.x) : -INF);
            const float mxy = warp_max(pending ? fmaxf(so.y, se.y) : -INF);
            const float mxz = warp_max(pending ? fmaxf(so.z, se.z) : -INF);
            const int leader = __ffs(shadow_lanes) - 1;
            const float3 pl = mk3(__shfl_sync(FULL, so.x, leader), __shfl_sync(FULL, so.y, leader),
                __shfl_sync(FULL, so.z, leader));
            float3 ell = lt.position - pl;
            const float ell_len = sqrtf(dot(ell, ell));
            constexpr int AXES = 5;
            float3 axis[AXES];
            float support[AXES];
            int axes = 0;
            if (ell_len > 1e-3f) {
                ell = ell * (1.0f / ell_len);
                const float kappa = lt.radius / ell_len;
                const float3 side = fabsf(ell.x) < 0.9f ? mk3(1.0f, 0.0f, 0.0f) : mk3(0.0f, 1.0f, 0.0f);
                const float3 u = normalize(cross(ell, side));
                const float3 v = cross(ell, u);
                axis[0] = u - ell * kappa;
                axis[1] = -u - ell * kappa;
                axis[2] = v - ell * kappa;
                axis[3] = -v - ell * kappa;
                axis[4] = -ell;
                axes = AXES;
#pragma unroll
                for (int k = 0; k < AXES; ++k)
                    support[k] = warp_max(pending ? fmaxf(dot(axis[k], so), dot(axis[k], se)) : -INF);
            }
            // Every instance of the world against the hull, 32 at a time: the candidates, in leaf order.
            const float light_scale = fabsf(lt.position.x) + fabsf(lt.position.y) + fabsf(lt.position.z) + lt.radius + 1.0f;
            __syncwarp();
            for (int base = 0; base < P; base += 32) {
                const int j = base + lane;
                bool scand = false;
                if (j < P) {
                    const float4 lo = __ldg(leaves + 2 * j), hi = __ldg(leaves + 2 * j + 1);
                    const float3 c = mk3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
                    const float3 h = mk3(0.5f * (hi.x - lo.x), 0.5f * (hi.y - lo.y), 0.5f * (hi.z - lo.z));
                    const float pad = 1e-4f * (light_scale + fabsf(c.x) + fabsf(c.y) + fabsf(c.z) + h.x + h.y + h.z);
                    scand = hi.x >= mnx - pad && lo.x <= mxx + pad && hi.y >= mny - pad && lo.y <= mxy + pad &&
                        hi.z >= mnz - pad && lo.z <= mxz + pad;
#pragma unroll
                    for (int k = 0; k < AXES; ++k) {
                        if (k < axes && dot(axis[k], c) - abs_dot(axis[k], h) >
                                support[k] + pad * (fabsf(axis[k].x) + fabsf(axis[k].y) + fabsf(axis[k].z)))
                            scand = false;
                    }
                }
                const unsigned cmask = __ballot_sync(FULL, scand);
                if (scand) cand_leaf[ncand + __popc(cmask & below)] = j;
                ncand += __popc(cmask);
            }
            __syncwarp();
            // The ray's own mesh first when the shade kernel found it starts on that body's side, or not at all when
            // it cannot meet it; any hit ends the ray whatever the order, so the answer is the same.
            const int self_code = pending ? a.shadow_self[T.pix] : -1;
            const int self = self_code >= 0 ? self_code >> 2 : -1;
            bool blocked = false;
            const float3 sinv = safe_inverse(sd);
            // Step -1 (when some lane has one): each lane's own mesh where it is walked first, from its leaf (leaf k
            // of the sorted leaves is node n - 1 + k); then the candidates in turn. One walk site, inlined.
            const bool self_first = self_code >= 0 && (self_code & 3) == 2;
            for (int c = __any_sync(FULL, self_first) ? -1 : 0; c < ncand; ++c) {
                const bool open = pending && !blocked;
                if (!__any_sync(FULL, open)) break;
                const float4 *leaf = c >= 0 ? leaves + 2 * cand_leaf[c]
                    : s.tlas + 2 * (static_cast<long long>(s.tlas_internal) + __ldg(s.leaf_of + (self_first ? self : 0)));
                const float4 lo = __ldg(leaf), hi = __ldg(leaf + 1);
                const int id = ~__float_as_int(lo.w);
                const bool walk = c >= 0 ? id != self : self_first;
                if (open && walk && box_entry(lo, hi, so, sinv, sdist) < NO_HIT) {
                    float tm = sdist, hu, hv;
                    int ht;
                    blocked = instance_walk_body<true>(s.inst, s.slot_bounds, s.slot_root, s.blas_pairs, s.tris,
                        s.slot_sphere, id, so, sd, tm, ht, hu, hv, max_steps, a.error_flag);
                }
            }
            if (pending && a.radiance) {
                if (blocked) a.radiance[T.pix] = a.pic_hit[T.pix];
            } else if (pending) {
                put_rgb(a.rgb, T.pix, blocked ? a.pic_code[T.pix] : __float_as_int(d4.w));
            }
        }
    }
}

// Shadow rays of worlds walked as packets (above TILE_MAX_INSTANCES instances), per 8 x 4 tile: the tile's
// pending shadow rays (those the shade kernel left) walk the world's tree together, a lane stopping at its first
// hit (packet_walk<true>); a lane leaves out its own mesh where the shade kernel found the ray cannot meet it.
// Neighbouring pixels' rays leave nearby points for the same light, so they enter nearly the same nodes.
template <int THREADS, int MIN_BLOCKS>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) shadow_packets_kernel(const __grid_constant__ SceneParams s,
    const RenderArgs a, int *counter, long long tiles, int tiles_x, int tiles_per_view, int fetch) {
    __shared__ WarpSmem<0> warp_smem[THREADS / 32];
    WarpSmem<0> &sm = warp_smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int max_steps = s.blas_node_count + 2;
    for (;;) {
        const long long first = fetch_tiles(counter, lane, fetch);
        if (first >= tiles) break;
        const long long last = first + fetch < tiles ? first + fetch : tiles;
        for (long long tile = first; tile < last; ++tile) {
            const TileAt T = tile_at(a, tile, tiles_x, tiles_per_view, lane);
            float4 o4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (T.pixel) o4 = a.shadow_o[T.pix];
            const bool pending = o4.w > 0.0f;
            if (!__any_sync(FULL, pending)) continue;
            float4 d4 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
            int self_code = -1;
            if (pending) {
                d4 = a.shadow_d[T.pix];
                self_code = a.shadow_self[T.pix];
            }
            const int skip = self_code >= 0 && (self_code & 3) == 1 ? self_code >> 2 : -1;
            float tmax = o4.w, hu = 0.0f, hv = 0.0f;
            int hit_inst = -1, hit_tri = -1;
            packet_walk<true>(s, sm, lane, T.world, pending, mk3(o4.x, o4.y, o4.z), mk3(d4.x, d4.y, d4.z), tmax,
                hit_inst, hit_tri, hu, hv, skip, max_steps, a.error_flag);
            const bool blocked = hit_inst >= 0;
            if (pending && a.radiance) {
                if (blocked) a.radiance[T.pix] = a.pic_hit[T.pix];
            } else if (pending) {
                put_rgb(a.rgb, T.pix, blocked ? a.pic_code[T.pix] : __float_as_int(d4.w));
            }
        }
    }
}

// Ray queries as warp packets (cast_ray, src/render_core.h:331-349): a warp takes 32 consecutive rays of one world
// and walks the world's tree as a packet (packet_walk: every node some lane's ray enters, visited once for all
// lanes, each lane entering only the instances its own ray enters), then each lane resolves its own hit. Rays
// from one sensor in scan order (a LiDAR's neighbouring beams) enter nearly the same nodes, so the warp's lanes
// share the walk instead of each walking alone; every ray still gets its own walk's closest hit (up to which of
// two equally distant hits is kept).
template <int THREADS, int MIN_BLOCKS>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) ray_packets_kernel(const __grid_constant__ SceneParams s,
    const RayArgs r, int *counter, long long groups, int groups_per_world) {
    __shared__ WarpSmem<0> warp_smem[THREADS / 32];
    WarpSmem<0> &sm = warp_smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int max_steps = s.blas_node_count + 2;
    for (;;) {
        const long long g = fetch_tiles(counter, lane, 1);
        if (g >= groups) break;
        const int world = static_cast<int>(g / groups_per_world);
        const int local = static_cast<int>(g % groups_per_world) * 32 + lane;
        const bool valid = local < r.rays_per_world;
        const long long i = static_cast<long long>(world) * r.rays_per_world + local;
        float3 o = mk3(0.0f, 0.0f, 0.0f), d = mk3(0.0f, 0.0f, 1.0f);
        bool live = false;
        if (valid) {
            o = mk3(__ldg(r.origins + 3 * i), __ldg(r.origins + 3 * i + 1), __ldg(r.origins + 3 * i + 2));
            d = mk3(__ldg(r.directions + 3 * i), __ldg(r.directions + 3 * i + 1), __ldg(r.directions + 3 * i + 2));
            const float len2 = dot(d, d);
            live = len2 > 1e-30f && len2 < 1e30f;  // compared with >, so a NaN direction is a miss too
            if (live) d = d * (1.0f / sqrtf(len2));
            else d = mk3(0.0f, 0.0f, 1.0f);
        }
        int best_sphere = -1;
        bool hit_floor = false;
        float tmax = live ? spheres_and_floor(s, o, d, best_sphere, hit_floor) : 0.0f;
        int hit_inst = -1, hit_tri = -1;
        float hu = 0.0f, hv = 0.0f;
        packet_walk<false>(s, sm, lane, world, live, o, d, tmax, hit_inst, hit_tri, hu, hv, -1, max_steps, r.error_flag);
        if (!valid) continue;
        const bool found = live && (hit_inst >= 0 || best_sphere >= 0 || hit_floor) && tmax <= r.max_distance;
        float3 normal = mk3(0.0f, 0.0f, 0.0f);
        DevMaterial mat{};
        int object = OBJECT_NONE;
        if (found) resolve(s, world, o + d * tmax, d, hit_inst, hit_tri, hu, hv, best_sphere, hit_floor, normal, mat, object);
        r.distance[i] = found ? tmax : __int_as_float(0x7f800000);
        r.normal[3 * i] = normal.x;
        r.normal[3 * i + 1] = normal.y;
        r.normal[3 * i + 2] = normal.z;
        r.object_id[i] = found ? object : OBJECT_NONE;
    }
}

template <class Kernel>
cudaError_t launch_tiles(Kernel kernel, int threads, const SceneParams &s, const RenderArgs &a, int *counter,
    long long tiles, int tiles_x, int tiles_per_view, int fetch, cudaStream_t stream) {
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    // Every SM full of resident warps, and no more warps than there are fetches of tiles.
    long long blocks = static_cast<long long>(sms) * per_sm;
    const long long needed = (tiles + fetch * (threads / 32) - 1) / (fetch * (threads / 32));
    if (blocks > needed) blocks = needed;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    kernel<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(s, a, counter, tiles, tiles_x, tiles_per_view, fetch);
    return cudaGetLastError();
}

template <int THREADS, int MIN_BLOCKS, int CAP>
cudaError_t launch_variant(const SceneParams &s, const RenderArgs &a, int *counter, const PersistentTuning &t,
    cudaStream_t stream, cudaEvent_t after_camera, cudaEvent_t after_shade) {
    const int fetch = t.tile_fetch;
    const int tiles_x = (a.width + TILE_W - 1) / TILE_W, tiles_y = (a.rows + TILE_H - 1) / TILE_H;
    const int tiles_per_view = tiles_x * tiles_y;
    const long long tiles = a.view_info ? a.total_tiles : static_cast<long long>(tiles_per_view) * a.views;
    const bool aov = a.depth || a.normal || a.object_id || a.hit_instance;
    cudaError_t e = cudaSuccess;
    auto mark = [&](cudaEvent_t ev) {
        if (e == cudaSuccess && ev) e = cudaEventRecord(ev, stream);
    };
    if (tiles == 0 || (!a.rgb && !aov)) {
        mark(after_camera);
        mark(after_shade);
        return e;
    }
    if (!a.basis_given) e = launch_prepare_cameras(a.cameras, a.views, a.camera_basis, stream);
    if constexpr (CAP > 0) {
        if (e == cudaSuccess && a.views > 0) {
            view_order_kernel<CAP><<<static_cast<unsigned>(a.views), 128, 0, stream>>>(s, a);
            e = cudaGetLastError();
        }
    }
    // Both kinds of camera ray: paired 4 x 4 tiles (pair_tile_at).
    const bool paired = t.tile_pairs && a.rgb && aov && (!a.view_info || a.view_pair_tile);
    if (e == cudaSuccess && paired) {
        const int ptx = (a.width + 3) / 4, pty = (a.rows + 3) / 4;
        const long long pair_tiles = a.view_info ? a.total_pair_tiles : static_cast<long long>(ptx) * pty * a.views;
        e = launch_tiles(camera_tiles_kernel<THREADS, MIN_BLOCKS, CAP, true>, THREADS, s, a, counter, pair_tiles, ptx,
            ptx * pty, fetch, stream);
    } else if (e == cudaSuccess) {
        e = launch_tiles(camera_tiles_kernel<THREADS, MIN_BLOCKS, CAP, false>, THREADS, s, a, counter, tiles, tiles_x,
            tiles_per_view, fetch, stream);
    }
    mark(after_camera);
    if (e != cudaSuccess || !a.rgb) {
        mark(after_shade);
        return e;
    }
    const long long pixels = a.view_info ? a.total_pixels : static_cast<long long>(a.views) * a.width * a.rows;
    int device = 0, sms = 0;
    e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    long long blocks = (pixels + 255) / 256;
    if (blocks > 32LL * sms) blocks = 32LL * sms;
    if (a.radiance) shade_kernel<true><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(s, a, pixels);
    else shade_kernel<false><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(s, a, pixels);
    e = cudaGetLastError();
    mark(after_shade);
    if (e != cudaSuccess || s.light_count != 1) return e;
    // Worlds too large for candidate lists: the shadow rays as warp packets over the world's tree (0.39 against
    // 0.41 ms as persistent-kernel jobs with lane refill on the large world's 1280 x 720 frame).
    if constexpr (CAP == 0) {
        return launch_tiles(shadow_packets_kernel<THREADS, MIN_BLOCKS>, THREADS, s, a, counter, tiles, tiles_x,
            tiles_per_view, fetch, stream);
    } else {
        return launch_tiles(shadow_tiles_kernel<THREADS, MIN_BLOCKS, CAP>, THREADS, s, a, counter, tiles, tiles_x,
            tiles_per_view, fetch, stream);
    }
}

}  // namespace

cudaError_t launch_rays_packets(const SceneParams &s, const RayArgs &r, int *counter, cudaStream_t stream) {
    if (r.count <= 0 || r.rays_per_world <= 0) return cudaSuccess;
    constexpr int THREADS = 128;
    auto kernel = ray_packets_kernel<THREADS, 9>;
    const int groups_per_world = (r.rays_per_world + 31) / 32;
    const long long groups = static_cast<long long>(groups_per_world) * (r.count / r.rays_per_world);
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, THREADS, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long blocks = static_cast<long long>(sms) * per_sm;
    const long long needed = (groups + THREADS / 32 - 1) / (THREADS / 32);
    if (blocks > needed) blocks = needed;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    kernel<<<static_cast<unsigned>(blocks), THREADS, 0, stream>>>(s, r, counter, groups, groups_per_world);
    return cudaGetLastError();
}

cudaError_t launch_render_tiles(const SceneParams &s, const RenderArgs &a, int *counter, const PersistentTuning &t,
    cudaStream_t stream, cudaEvent_t after_camera, cudaEvent_t after_shade) {
    // (threads per CTA, register budget) -> the instantiation with that budget, and the candidate lists'
    // capacity: 32 for worlds of up to 32 instances, else TILE_MAX_INSTANCES; larger worlds walk their tree
    // as a packet (capacity 0).
    if (s.instance_count > 0 && s.per_world > TILE_MAX_INSTANCES) {
        if (t.threads == 128 && t.registers == 64) return launch_variant<128, 8, 0>(s, a, counter, t, stream, after_camera, after_shade);
        if (t.threads == 128 && t.registers == 56) return launch_variant<128, 9, 0>(s, a, counter, t, stream, after_camera, after_shade);
        if (t.threads == 128 && t.registers == 48) return launch_variant<128, 10, 0>(s, a, counter, t, stream, after_camera, after_shade);
        if (t.threads == 128 && t.registers == 80) return launch_variant<128, 6, 0>(s, a, counter, t, stream, after_camera, after_shade);
        if (t.threads == 256 && t.registers == 64) return launch_variant<256, 4, 0>(s, a, counter, t, stream, after_camera, after_shade);
        return cudaErrorInvalidValue;
    }
    const bool small = s.per_world <= 32;
    if (t.threads == 128 && t.registers == 64)
        return small ? launch_variant<128, 8, 32>(s, a, counter, t, stream, after_camera, after_shade)
                     : launch_variant<128, 8, TILE_MAX_INSTANCES>(s, a, counter, t, stream, after_camera, after_shade);
    if (t.threads == 128 && t.registers == 56)
        return small ? launch_variant<128, 9, 32>(s, a, counter, t, stream, after_camera, after_shade)
                     : launch_variant<128, 9, TILE_MAX_INSTANCES>(s, a, counter, t, stream, after_camera, after_shade);
    if (t.threads == 128 && t.registers == 48)
        return small ? launch_variant<128, 10, 32>(s, a, counter, t, stream, after_camera, after_shade)
                     : launch_variant<128, 10, TILE_MAX_INSTANCES>(s, a, counter, t, stream, after_camera, after_shade);
    if (t.threads == 128 && t.registers == 80)
        return small ? launch_variant<128, 6, 32>(s, a, counter, t, stream, after_camera, after_shade)
                     : launch_variant<128, 6, TILE_MAX_INSTANCES>(s, a, counter, t, stream, after_camera, after_shade);
    if (t.threads == 256 && t.registers == 64)
        return small ? launch_variant<256, 4, 32>(s, a, counter, t, stream, after_camera, after_shade)
                     : launch_variant<256, 4, TILE_MAX_INSTANCES>(s, a, counter, t, stream, after_camera, after_shade);
    return cudaErrorInvalidValue;
}

}  // namespace ngb
