// Device functions shared by the trace kernels: intersection, traversal of the reference's node layout,
// surface resolve and shading (src/mesh_dev.h, src/render_core.h, src/device_scene.h, src/geom_dev.h).
#pragma once

#include "device.cuh"

namespace ngb {
namespace tr {
namespace {


// 1/x that never produces infinity (src/mesh_dev.h:58-61).
__device__ __forceinline__ float3 safe_inverse(float3 d) {
    const float x = fabsf(d.x) < 1e-12f ? copysignf(1e-12f, d.x) : d.x;
    const float y = fabsf(d.y) < 1e-12f ? copysignf(1e-12f, d.y) : d.y;
    const float z = fabsf(d.z) < 1e-12f ? copysignf(1e-12f, d.z) : d.z;
    return mk3(recip(x), recip(y), recip(z));
}

// The largest and smallest of three (sm_100's three-input max.f32 / min.f32: max(max(a, b), c), one
// instruction instead of two).
__device__ __forceinline__ float max3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Slab test (src/mesh_dev.h:66-74): where the ray enters the box, or NO_HIT. The entry is the largest of the
// three near planes and 0, the exit the smallest of the three far planes and tmax; no operand is a NaN (the
// inverse direction is finite), so grouping the maxima and minima in threes gives the reference's values.
__device__ __forceinline__ float box_entry(float4 lo, float4 hi, float3 o, float3 inv_d, float tmax) {
    const float tx0 = (lo.x - o.x) * inv_d.x, tx1 = (hi.x - o.x) * inv_d.x;
    const float ty0 = (lo.y - o.y) * inv_d.y, ty1 = (hi.y - o.y) * inv_d.y;
    const float tz0 = (lo.z - o.z) * inv_d.z, tz1 = (hi.z - o.z) * inv_d.z;
    const float tn = max3(fminf(tx0, tx1), fminf(ty0, ty1), fmaxf(fminf(tz0, tz1), 0.0f));
    const float tf = min3(fmaxf(tx0, tx1), fmaxf(ty0, ty1), fminf(fmaxf(tz0, tz1), tmax));
    return tn <= tf ? tn : NO_HIT;
}

// Two-sided Moller-Trumbore (src/mesh_dev.h:80-99).
__device__ __forceinline__ bool triangle_hit(const float4 *tris, int i, float3 o, float3 d, float tmax, float &t,
    float &bu, float &bv) {
    const float3 v0 = xyz(__ldg(tris + 3 * i));
    const float3 e1 = xyz(__ldg(tris + 3 * i + 1));
    const float3 e2 = xyz(__ldg(tris + 3 * i + 2));
    const float3 p = cross(d, e2);
    const float det = dot(e1, p);
    if (fabsf(det) < 1e-14f) return false;
    const float inv_det = recip(det);
    const float3 s = o - v0;
    const float u = dot(s, p) * inv_det;
    if (u < 0.0f || u > 1.0f) return false;
    const float3 q = cross(s, e1);
    const float v = dot(d, q) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, q) * inv_det;
    bu = u;
    bv = v;
    return t > 0.0f && t < tmax;
}

struct InstanceRec {
    float4 r0, r1, r2;
    int blas_root;
};

__device__ __forceinline__ InstanceRec load_instance(const float4 *inst, int id) {
    InstanceRec r;
    r.r0 = __ldg(inst + 4 * id);
    r.r1 = __ldg(inst + 4 * id + 1);
    r.r2 = __ldg(inst + 4 * id + 2);
    r.blas_root = __float_as_int(__ldg(inst + 4 * id + 3).x);
    return r;
}

// World to mesh space (src/mesh_dev.h:164-171). The direction is not renormalised, so t is shared.
__device__ __forceinline__ float3 to_local_point(const InstanceRec &r, float3 p) {
    return mk3(dot(xyz(r.r0), p) + r.r0.w, dot(xyz(r.r1), p) + r.r1.w, dot(xyz(r.r2), p) + r.r2.w);
}
__device__ __forceinline__ float3 to_local_dir(const InstanceRec &r, float3 d) {
    return mk3(dot(xyz(r.r0), d), dot(xyz(r.r1), d), dot(xyz(r.r2), d));
}

// One mesh's tree (traverse<false>, src/mesh_dev.h:113-159). Closest: lowers tmax and records the hit.
// Any: returns true at the first hit closer than tmax. Nearer child first; the farther one is pushed with
// its entry distance and dropped at pop time once a closer hit is known.
template <bool Any>
__device__ __forceinline__ bool blas_walk(const float4 *blas, const float4 *tris, int root, float3 o, float3 d,
    float &tmax, int instance, int &hit_instance, int &hit_triangle, float &hu, float &hv, bool &found, int max_steps,
    int *err) {
    const float3 inv_d = safe_inverse(d);
    if (box_entry(__ldg(blas + 2 * root), __ldg(blas + 2 * root + 1), o, inv_d, tmax) >= NO_HIT) return false;
    int stack[BLAS_STACK];
    float stack_t[BLAS_STACK];
    int sp = 0, node = root;
    for (int steps = 0;; ++steps) {
        if (steps > max_steps) {  // only a malformed tree gets here
            *err = 2;
            return false;
        }
        const float4 n0 = __ldg(blas + 2 * node), n1 = __ldg(blas + 2 * node + 1);
        const int w0 = __float_as_int(n0.w), w1 = __float_as_int(n1.w);
        bool descended = false;
        if (w1 > 0) {
            for (int j = w0; j < w0 + w1; ++j) {
                float t, bu, bv;
                if (triangle_hit(tris, j, o, d, tmax, t, bu, bv)) {
                    if (Any) return true;
                    tmax = t;
                    hit_instance = instance;
                    hit_triangle = j;
                    hu = bu;
                    hv = bv;
                    found = true;
                }
            }
        } else {
            const int a = w0, right = w0 + 1;
            const float dl = box_entry(__ldg(blas + 2 * a), __ldg(blas + 2 * a + 1), o, inv_d, tmax);
            const float dr = box_entry(__ldg(blas + 2 * right), __ldg(blas + 2 * right + 1), o, inv_d, tmax);
            if (dl < NO_HIT || dr < NO_HIT) {
                const bool left_first = dl <= dr;
                const float far_t = left_first ? dr : dl;
                if (far_t < NO_HIT) {
                    if (sp >= BLAS_STACK) {
                        *err = 1;
                        return false;
                    }
                    stack[sp] = left_first ? right : a;
                    stack_t[sp] = far_t;
                    ++sp;
                }
                node = left_first ? a : right;
                descended = true;
            }
        }
        if (descended) continue;
        while (sp > 0 && stack_t[sp - 1] >= tmax) --sp;
        if (sp == 0) return false;
        node = stack[--sp];
    }
}

// A world's tree over its instances (traverse<true>) with mesh_intersect / mesh_occluded's leaf
// (src/mesh_dev.h:177-227). Returns, for Any, whether something blocks; otherwise whether a hit was found.
template <bool Any>
__device__ __noinline__ bool mesh_query(const SceneParams &s, int world, float3 o, float3 d, float &tmax,
    int &hit_instance, int &hit_triangle, float &hu, float &hv, int *err) {
    const float4 *tlas = s.tlas;
    const float3 inv_d = safe_inverse(d);
    const int root = __ldg(s.roots + world);
    bool found = false;
    if (root < 0) return false;  // a world without instances
    if (box_entry(__ldg(tlas + 2 * root), __ldg(tlas + 2 * root + 1), o, inv_d, tmax) >= NO_HIT) return false;
    int stack[TLAS_STACK];
    float stack_t[TLAS_STACK];
    int sp = 0, node = root;
    const int max_steps = 2 * s.per_world + 2;
    for (int steps = 0;; ++steps) {
        if (steps > max_steps) {  // only a malformed tree gets here
            *err = 2;
            return Any ? false : found;
        }
        const float4 n0 = __ldg(tlas + 2 * node), n1 = __ldg(tlas + 2 * node + 1);
        const int w0 = __float_as_int(n0.w), w1 = __float_as_int(n1.w);
        bool descended = false;
        if (w0 < 0) {
            const int id = ~w0;
            const InstanceRec r = load_instance(s.inst, id);
            if (blas_walk<Any>(s.blas, s.tris, r.blas_root, to_local_point(r, o), to_local_dir(r, d), tmax, id,
                    hit_instance, hit_triangle, hu, hv, found, s.blas_node_count, err))
                return true;
        } else {
            const int a = w0, right = w1;
            const float dl = box_entry(__ldg(tlas + 2 * a), __ldg(tlas + 2 * a + 1), o, inv_d, tmax);
            const float dr = box_entry(__ldg(tlas + 2 * right), __ldg(tlas + 2 * right + 1), o, inv_d, tmax);
            if (dl < NO_HIT || dr < NO_HIT) {
                const bool left_first = dl <= dr;
                const float far_t = left_first ? dr : dl;
                if (far_t < NO_HIT) {
                    if (sp >= TLAS_STACK) {
                        *err = 1;
                        return found;
                    }
                    stack[sp] = left_first ? right : a;
                    stack_t[sp] = far_t;
                    ++sp;
                }
                node = left_first ? a : right;
                descended = true;
            }
        }
        if (descended) continue;
        while (sp > 0 && stack_t[sp - 1] >= tmax) --sp;
        if (sp == 0) return Any ? false : found;
        node = stack[--sp];
    }
}

struct Hit {
    float3 point;
    float3 normal;
    DevMaterial material;
    float t;
    int object;
    int instance;  // the mesh hit's record, -1 for a sphere or the floor
    int triangle;
    float u, v;
};

__device__ __forceinline__ bool sphere_hit(const DevSphere &sp, float3 origin, float3 dir, float &t) {
    const float3 L = sp.center - origin;
    const float tca = dot(L, dir);
    const float r2 = sp.radius * sp.radius;
    const float d2 = dot(L, L) - tca * tca;
    if (d2 > r2) return false;
    const float thc = sqrtf(r2 - d2);
    t = tca - thc;
    if (t < 0.0f) t = tca + thc;
    return t >= 0.0f;
}

__device__ __forceinline__ bool floor_hit(const DevPlane &f, float3 origin, float3 dir, float limit, float &out) {
    if (!(fabsf(dir.y) > 1e-3f)) return false;
    const float d = (f.y - origin.y) / dir.y;
    if (!(d > 0.0f && d < limit)) return false;
    const float3 pt = origin + dir * d;
    if (fabsf(pt.x) < f.hx && pt.z > f.zmin && pt.z < f.zmax) {
        out = d;
        return true;
    }
    return false;
}

// The shading normal at a triangle hit, facing the ray (src/mesh_dev.h:238-262, without textures).
__device__ __forceinline__ float3 mesh_surface(const SceneParams &s, int instance, int triangle, float hu, float hv,
    float3 dir) {
    const InstanceRec r = load_instance(s.inst, instance);
    const float3 r0 = xyz(r.r0), r1 = xyz(r.r1), r2 = xyz(r.r2);
    const float3 nl = cross(xyz(__ldg(s.tris + 3 * triangle + 1)), xyz(__ldg(s.tris + 3 * triangle + 2)));
    float3 geometric = normalize(r0 * nl.x + r1 * nl.y + r2 * nl.z);
    if (dot(geometric, dir) > 0.0f) geometric = -geometric;
    float3 normal = geometric;
    if (s.attrs == nullptr) return normal;
    const float4 a0 = __ldg(s.attrs + 4 * triangle), a1 = __ldg(s.attrs + 4 * triangle + 1);
    const float4 a2 = __ldg(s.attrs + 4 * triangle + 2), a3 = __ldg(s.attrs + 4 * triangle + 3);
    const float w0 = 1.0f - hu - hv;
    if (__float_as_int(a3.w) & 1) {
        const float3 n = xyz(a0) * w0 + xyz(a1) * hu + xyz(a2) * hv;
        if (dot(n, n) > 1e-12f) {
            const float3 smooth = normalize(r0 * n.x + r1 * n.y + r2 * n.z);
            normal = dot(smooth, geometric) < 0.0f ? -smooth : smooth;
        }
    }
    return normal;
}

// Closest hit over spheres, the floor and the world's meshes (src/render_core.h:78-143).
__device__ __forceinline__ bool scene_intersect(const SceneParams &s, int world, float3 origin, float3 dir, Hit &hit, int *err) {
    float best = 1e30f;
    int best_sphere = -1;
    for (int i = 0; i < s.sphere_count; ++i) {
        float t;
        if (sphere_hit(s.spheres[i], origin, dir, t) && t < best) {
            best = t;
            best_sphere = i;
        }
    }
    bool hit_floor = false;
    {
        float d;
        if (floor_hit(s.floor, origin, dir, best, d)) {
            best = d;
            hit_floor = true;
        }
    }
    int best_instance = -1, best_triangle = -1;
    float bu = 0.0f, bv = 0.0f;
    if (s.instance_count > 0 &&
        mesh_query<false>(s, world, origin, dir, best, best_instance, best_triangle, bu, bv, err)) {
        best_sphere = -1;
        hit_floor = false;
    } else {
        best_instance = -1;
    }
    if (best_sphere < 0 && !hit_floor && best_instance < 0) return false;
    hit.t = best;
    hit.point = origin + dir * best;
    hit.instance = -1;
    hit.triangle = -1;
    hit.u = hit.v = 0.0f;
    if (best_instance >= 0) {
        hit.normal = mesh_surface(s, best_instance, best_triangle, bu, bv, dir);
        hit.material = s.slot_material[table_of(s, best_instance, world)];
        hit.object = OBJECT_INSTANCE + (best_instance - world_first_of(s, world));
        hit.instance = best_instance;
        hit.triangle = best_triangle;
        hit.u = bu;
        hit.v = bv;
    } else if (hit_floor) {
        hit.object = OBJECT_FLOOR;
        hit.normal = mk3(0.0f, 1.0f, 0.0f);
        hit.material = s.floor.m;
        const int cx = static_cast<int>(floorf(hit.point.x * s.floor.checker));
        const int cz = static_cast<int>(floorf(hit.point.z * s.floor.checker));
        const float3 tint = ((cx + cz) & 1) ? mk3(1.0f, 1.0f, 1.0f) : mk3(1.0f, 0.7f, 0.3f);
        hit.material.diffuse_color = tint * 0.3f;
    } else {
        hit.normal = normalize(hit.point - s.spheres[best_sphere].center);
        hit.material = s.spheres[best_sphere].m;
        hit.object = OBJECT_SPHERE + best_sphere;
    }
    return true;
}

// Any hit closer than max_dist (src/render_core.h:146-161).
__device__ __forceinline__ bool scene_occluded(const SceneParams &s, int world, float3 origin, float3 dir, float max_dist, int *err) {
    for (int i = 0; i < s.sphere_count; ++i) {
        float t;
        if (sphere_hit(s.spheres[i], origin, dir, t) && t < max_dist) return true;
    }
    {
        float d;
        if (floor_hit(s.floor, origin, dir, max_dist, d)) return true;
    }
    if (s.instance_count <= 0) return false;
    float tmax = max_dist, hu, hv;
    int hi, ht;
    return mesh_query<true>(s, world, origin, dir, tmax, hi, ht, hu, hv, err);
}

// How much of a light reaches a point (src/device_scene.h:98-111).
__device__ __forceinline__ float light_factor(const DevLight &l, float3 towards, float d) {
    float f = 1.0f;
    if (l.falloff > 0.0f) {
        const float q = d / l.falloff;
        f = 1.0f / (1.0f + q * q);
    }
    if (l.cos_outer > -1.5f) {
        const float c = -(l.direction.x * towards.x + l.direction.y * towards.y + l.direction.z * towards.z);
        const float t = fminf(fmaxf((c - l.cos_outer) / fmaxf(l.cos_inner - l.cos_outer, 1e-6f), 0.0f), 1.0f);
        f *= t * t * (3.0f - 2.0f * t);
    }
    return f;
}

__device__ __forceinline__ float3 offset_origin(float3 p, float3 n, float3 dir) {
    return p + n * (dot(dir, n) < 0.0f ? -1e-3f : 1e-3f);
}

// Classic shading with mirror bounces (src/render_core.h:202-245).
__device__ __forceinline__ float3 trace(const SceneParams &s, int world, float3 origin, float3 dir, uint32_t &rng, int *err) {
    float3 radiance = mk3(0.0f, 0.0f, 0.0f);
    float throughput = 1.0f;
    for (int depth = 0;; ++depth) {
        Hit hit;
        if (depth > 4 || !scene_intersect(s, world, origin, dir, hit, err)) {
            const float t = saturate(dot(dir, s.env_up) * 0.5f + 0.5f);
            const float3 sky = (s.env_color_down + (s.env_color_up - s.env_color_down) * t) * s.env_intensity;
            radiance = radiance + sky * throughput;
            break;
        }
        float3 diffuse = mk3(0.0f, 0.0f, 0.0f), specular = mk3(0.0f, 0.0f, 0.0f);
        for (int i = 0; i < s.light_count; ++i) {
            const DevLight &L = s.lights[i];
            // sample_sphere_light / random_unit_vector (src/geom_dev.h:136-152): always two draws.
            const float z = 1.0f - 2.0f * rand_float(rng);
            const float rad = sqrtf(fmaxf(0.0f, 1.0f - z * z));
            const float phi = 6.28318530718f * rand_float(rng);
            const float3 lp = L.position + mk3(rad * cosf(phi), rad * sinf(phi), z) * L.radius;
            const float3 to_light = lp - hit.point;
            const float light_distance = sqrtf(dot(to_light, to_light));
            const float3 light_dir = to_light * recip(light_distance);
            const float strength = L.intensity * light_factor(L, light_dir, light_distance);
            if (strength <= 0.0f) continue;
            if (scene_occluded(s, world, offset_origin(hit.point, hit.normal, light_dir), light_dir, light_distance, err))
                continue;
            const float3 lit = L.color * strength;
            diffuse = diffuse + lit * fmaxf(0.0f, dot(light_dir, hit.normal));
            specular = specular + lit * powf(fmaxf(0.0f, dot(reflect(light_dir, hit.normal), dir)), hit.material.exponent);
        }
        const float3 direct = hit.material.diffuse_color * (diffuse * hit.material.kd) + specular * hit.material.ks;
        radiance = radiance + (direct + hit.material.diffuse_color * (s.ambient * hit.material.kd)) * throughput;
        throughput *= hit.material.kr;
        if (throughput < 1e-3f) break;
        dir = reflect(dir, hit.normal);
        origin = offset_origin(hit.point, hit.normal, dir);
    }
    return radiance;
}

__device__ __forceinline__ float srgb_channel(float v) {
    const float x = saturate(v);
    return x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
}

__device__ __forceinline__ uint8_t to_byte(float c) { return static_cast<uint8_t>(saturate(c) * 255.0f + 0.5f); }

// The sRGB byte of a linear value, exactly as the host's powf makes it (src/geom_dev.h:169-176,
// render_core.h:280): a guess from the fast approximate power, then moved to the k with
// table[k] <= v < table[k + 1] (the table holds each byte's first float, made on the host and checked
// against every float of [0, 1]). A NaN stays at 0, as saturate makes it.
__device__ __forceinline__ uint8_t srgb_byte(const float *table, float v) {
    const float x = saturate(v);
    const float c = x <= 0.0031308f ? 12.92f * x : 1.055f * __powf(x, 1.0f / 2.4f) - 0.055f;
    int k = static_cast<int>(saturate(c) * 255.0f + 0.5f);
    while (k < 255 && v >= __ldg(table + k + 1)) ++k;
    while (k > 0 && v < __ldg(table + k)) --k;
    return static_cast<uint8_t>(k);
}


// The camera ray through image point (px, py) (camera_ray, src/device_scene.h:114-119): the tangent-plane offsets, then the
// direction normalised.
__device__ __forceinline__ float3 camera_dir(float3 right, float3 up, float3 fwd, float px, float py, float fw, float fh,
    float fov_scale, float aspect) {
    const float sx = (2.0f * px / fw - 1.0f) * fov_scale * aspect;
    const float sy = -(2.0f * py / fh - 1.0f) * fov_scale;
    return normalize(right * sx + up * sy + fwd);
}

// The radiance of a hit with these light sums, as trace computes it for a path of one bounce
// (src/render_core.h:234-236, radiance and throughput starting at 0 and 1).
__device__ __forceinline__ float3 radiance_of(const DevMaterial &m, float ambient, float3 diffuse, float3 specular) {
    const float3 direct = m.diffuse_color * (diffuse * m.kd) + specular * m.ks;
    return mk3(0.0f, 0.0f, 0.0f) + (direct + m.diffuse_color * (ambient * m.kd)) * 1.0f;
}

// The bytes write_rgb stores for a radiance, packed r | g << 8 | b << 16.
__device__ __forceinline__ int rgb_packed(const float *table, float3 radiance) {
    float3 sum = mk3(0.0f, 0.0f, 0.0f) + radiance;
    sum = sum * (1.0f / 1.0f);
    return srgb_byte(table, sum.x) | (srgb_byte(table, sum.y) << 8) | (srgb_byte(table, sum.z) << 16);
}

// sample_pixel's average of one sample, sRGB, bytes (src/render_core.h:248-283).
__device__ __forceinline__ void write_rgb(const float *table, uint8_t *rgb, long long pix, float3 radiance) {
    float3 sum = mk3(0.0f, 0.0f, 0.0f) + radiance;
    sum = sum * (1.0f / 1.0f);
    uint8_t *o = rgb + 3 * static_cast<size_t>(pix);
    o[0] = srgb_byte(table, sum.x);
    o[1] = srgb_byte(table, sum.y);
    o[2] = srgb_byte(table, sum.z);
}

// Views of uneven sizes (view_info: per view width, height, first pixel, first tile): the last view whose
// first tile (by_tile) or first pixel is at most at.
__device__ __forceinline__ int view_of(const int4 *info, int views, long long at, bool by_tile) {
    int lo = 0, hi = views - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int4 v = __ldg(info + mid);
        if ((by_tile ? v.w : v.z) <= at) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace
}  // namespace tr
}  // namespace ngb
