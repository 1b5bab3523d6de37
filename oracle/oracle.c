/*
 * TEST INFRASTRUCTURE ONLY -- the oracle (see oracle.h). Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, and only as the checker.
 *
 * Every function cites the reference file:line it restates. Arithmetic is IEEE single precision in the
 * reference's source order; the build uses -ffp-contract=off so no multiply-add is fused.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

/* ------------------------------------------------------------------------------------- vector math -- */
/* src/geom_dev.h:18-62, host branch (NG_BACKEND_CPU). */

typedef struct {
    float x, y, z;
} f3;

static inline f3 mk(float x, float y, float z) {
    f3 r = {x, y, z};
    return r;
}
static inline f3 add3(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub3(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 mul3(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline f3 muls(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline f3 neg3(f3 a) { return mk(-a.x, -a.y, -a.z); }
static inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 cross3(f3 a, f3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
/* geom_dev.h:45-51: the host computes v * (1 / sqrt(v.v)). */
static inline f3 normalize3(f3 v) { return muls(v, 1.0f / sqrtf(dot3(v, v))); }
static inline float saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); } /* geom_dev.h:77-83 */
static inline f3 reflect3(f3 i, f3 n) { return sub3(i, muls(n, 2.0f * dot3(i, n))); } /* geom_dev.h:97 */
static inline f3 lerp3(f3 a, f3 b, float t) { return add3(a, muls(sub3(b, a), t)); }   /* geom_dev.h:62 */

/* --------------------------------------------------------------------------------------------- rng -- */
/* src/geom_dev.h:110-152. */

static inline uint32_t pcg_hash(uint32_t x) {
    const uint32_t state = x * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
static inline uint32_t make_rng(uint32_t pixel, uint32_t frame) { return pcg_hash(pixel ^ pcg_hash(frame + 1u)); }
static inline float rand_float(uint32_t *r) {
    *r = pcg_hash(*r);
    return (float)(*r) * 2.3283064365386963e-10f;
}
static inline f3 random_unit_vector(uint32_t *r) {
    const float z = 1.0f - 2.0f * rand_float(r);
    const float rad = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    const float phi = 6.28318530718f * rand_float(r);
    return mk(rad * cosf(phi), rad * sinf(phi), z);
}

/* -------------------------------------------------------------------------------------------- types -- */

typedef struct {
    f3 diffuse_color;
    float kd, ks, kr, exponent, roughness, metallic;
    f3 emission;
    float transmission, ior;
} mat_t;

typedef struct {
    f3 center;
    float radius;
    mat_t m;
} sphere_t;

/* device_scene.h:223-232, converted as to_device does (device_scene.h:265-272). */
typedef struct {
    f3 position;
    float intensity, radius, falloff;
    f3 direction;
    float cos_outer, cos_inner;
    f3 color;
} light_t;

typedef struct {
    float y, hx, zmin, zmax, checker;
    mat_t m;
} plane_t;

typedef struct { /* bvh::Node, src/bvh.h:30-35 */
    float lo[3];
    int32_t a;
    float hi[3];
    int32_t count;
} bnode_t;

typedef struct { /* bvh::TlasNode, src/bvh.h:44-49 */
    float lo[3];
    int32_t left;
    float hi[3];
    int32_t right;
} tnode_t;

typedef struct {
    float inv[12];
    int32_t blas_root;
} inst_t;

struct orc_scene {
    int W, H, worlds, cpw, P, n;
    sphere_t spheres[NGB_MAX_SPHERES];
    int nsph;
    light_t lights[NGB_MAX_LIGHTS];
    int nlig;
    plane_t floor;
    f3 env_up, env_cu, env_cd;
    float env_int, ambient;
    /* meshes */
    int mesh_count, blas_count, tri_count;
    bnode_t *blas;
    float *tris;        /* 12 per packed triangle */
    float *attrs;       /* 16 per packed triangle, or NULL */
    int32_t *tri_index; /* packed triangle -> index in its own mesh */
    int32_t *mesh_root;
    float *mesh_bounds; /* 6 per mesh */
    /* what each slot of a world holds */
    int32_t *slot_mesh;
    mat_t *slot_mat;
    /* per build */
    float *matrices;
    inst_t *inst;
    float *aabb;
    uint64_t *keys;
    int32_t *sorted_ids;
    uint64_t *sorted_keys;
    tnode_t *tlas;
    int32_t *roots;
    /* bodies */
    int bound, bpw;
    int32_t *boi;
    float *lpose, *lscale;
    double trav_bytes, trav_rays;
};

static mat_t to_mat(const ngb_material *m) {
    mat_t r;
    r.diffuse_color = mk(m->diffuse_color.x, m->diffuse_color.y, m->diffuse_color.z);
    r.kd = m->diffuse_albedo;
    r.ks = m->specular_albedo;
    r.kr = m->reflectivity;
    r.exponent = m->specular_exponent;
    r.roughness = m->roughness;
    r.metallic = m->metallic;
    r.emission = mk(m->emission.x, m->emission.y, m->emission.z);
    r.transmission = m->transmission;
    r.ior = m->ior;
    return r;
}

/* ------------------------------------------------------------------------ bottom-level tree build -- */
/* src/bvh.cpp:9-174, with std::min/std::max's exact semantics (b < a ? b : a, a < b ? b : a). */

#define BINS 16
#define MAX_DEPTH_BVH 60

typedef struct {
    float lo[3], hi[3];
} aabb_t;

static inline float smin(float a, float b) { return (b < a) ? b : a; }
static inline float smax(float a, float b) { return (a < b) ? b : a; }

static aabb_t empty_aabb(void) {
    aabb_t b;
    for (int i = 0; i < 3; ++i) {
        b.lo[i] = INFINITY;
        b.hi[i] = -INFINITY;
    }
    return b;
}
static void grow(aabb_t *box, const aabb_t *o) {
    for (int i = 0; i < 3; ++i) {
        box->lo[i] = smin(box->lo[i], o->lo[i]);
        box->hi[i] = smax(box->hi[i], o->hi[i]);
    }
}
static float surface_area(const aabb_t *b) {
    const float dx = b->hi[0] - b->lo[0], dy = b->hi[1] - b->lo[1], dz = b->hi[2] - b->lo[2];
    if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

typedef struct {
    int node;
    uint32_t begin, end;
    int depth;
} task_t;

static int bin_of(float c, float lo, float scale) {
    const int b = (int)((c - lo) * scale);
    return b < BINS - 1 ? b : BINS - 1;
}

/* libstdc++'s std::partition for bidirectional iterators (the overload a pointer range takes). */
static uint32_t *partition_bins(uint32_t *first, uint32_t *last, const float (*centroid)[3], int axis, float lo,
    float scale, int best_bin) {
    for (;;) {
        for (;;) {
            if (first == last) return first;
            if (bin_of(centroid[*first][axis], lo, scale) <= best_bin) ++first;
            else break;
        }
        --last;
        for (;;) {
            if (first == last) return first;
            if (!(bin_of(centroid[*last][axis], lo, scale) <= best_bin)) --last;
            else break;
        }
        const uint32_t t = *first;
        *first = *last;
        *last = t;
        ++first;
    }
}

/* bvh::build (src/bvh.cpp:46-174). Returns the node count; *nodes and order are malloc'ed/filled. */
static int bvh_build(const aabb_t *bounds, uint32_t n, int max_leaf, bnode_t **out_nodes, uint32_t *order) {
    if (n == 0) {
        *out_nodes = NULL;
        return 0;
    }
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    float (*centroid)[3] = malloc(sizeof(float[3]) * n);
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) centroid[i][k] = 0.5f * (bounds[i].lo[k] + bounds[i].hi[k]);
    bnode_t *nodes = calloc(2 * (size_t)n, sizeof(bnode_t));
    int node_count = 1;
    task_t *tasks = malloc(sizeof(task_t) * (2 * (size_t)n + 2));
    int ntask = 0;
    tasks[ntask++] = (task_t){0, 0, n, 0};
    while (ntask > 0) {
        const task_t task = tasks[--ntask];
        const uint32_t count = task.end - task.begin;
        uint32_t *prims = order + task.begin;
        aabb_t box = empty_aabb(), cbox = empty_aabb();
        for (uint32_t i = 0; i < count; ++i) {
            grow(&box, &bounds[prims[i]]);
            for (int k = 0; k < 3; ++k) {
                cbox.lo[k] = smin(cbox.lo[k], centroid[prims[i]][k]);
                cbox.hi[k] = smax(cbox.hi[k], centroid[prims[i]][k]);
            }
        }
        bnode_t node;
        memset(&node, 0, sizeof(node));
        for (int k = 0; k < 3; ++k) {
            node.lo[k] = box.lo[k];
            node.hi[k] = box.hi[k];
        }
        int best_axis = -1, best_bin = 0;
        float best_cost = INFINITY;
        if (count > 1) {
            for (int axis = 0; axis < 3; ++axis) {
                const float extent = cbox.hi[axis] - cbox.lo[axis];
                if (!(extent > 0.0f)) continue;
                const float scale = (float)BINS / extent;
                int bin_count[BINS] = {0};
                aabb_t bin_box[BINS];
                for (int b = 0; b < BINS; ++b) bin_box[b] = empty_aabb();
                for (uint32_t i = 0; i < count; ++i) {
                    const int b = bin_of(centroid[prims[i]][axis], cbox.lo[axis], scale);
                    ++bin_count[b];
                    grow(&bin_box[b], &bounds[prims[i]]);
                }
                float right_area[BINS - 1];
                int right_count[BINS - 1];
                aabb_t acc = empty_aabb();
                int running = 0;
                for (int i = BINS - 1; i >= 1; --i) {
                    grow(&acc, &bin_box[i]);
                    running += bin_count[i];
                    right_area[i - 1] = surface_area(&acc);
                    right_count[i - 1] = running;
                }
                acc = empty_aabb();
                running = 0;
                for (int i = 0; i < BINS - 1; ++i) {
                    grow(&acc, &bin_box[i]);
                    running += bin_count[i];
                    if (running == 0 || right_count[i] == 0) continue;
                    const float cost = (float)running * surface_area(&acc) + (float)right_count[i] * right_area[i];
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = axis;
                        best_bin = i;
                    }
                }
            }
        }
        const float leaf_cost = (float)count * surface_area(&box);
        const float split_cost = 1.0f * surface_area(&box) + best_cost;
        const int small = count <= (uint32_t)max_leaf;
        if (count == 1 || task.depth >= MAX_DEPTH_BVH || (small && (best_axis < 0 || leaf_cost <= split_cost))) {
            node.a = (int32_t)task.begin;
            node.count = (int32_t)count;
            nodes[task.node] = node;
            continue;
        }
        uint32_t mid;
        if (best_axis >= 0) {
            const float extent = cbox.hi[best_axis] - cbox.lo[best_axis];
            const float scale = (float)BINS / extent;
            const uint32_t *p = partition_bins(prims, prims + count, (const float (*)[3])centroid, best_axis,
                cbox.lo[best_axis], scale, best_bin);
            mid = task.begin + (uint32_t)(p - prims);
            if (mid == task.begin || mid == task.end) mid = task.begin + count / 2;
        } else {
            mid = task.begin + count / 2;
        }
        const int left = node_count;
        node_count += 2;
        node.a = left;
        node.count = 0;
        nodes[task.node] = node;
        tasks[ntask++] = (task_t){left + 1, mid, task.end, task.depth + 1};
        tasks[ntask++] = (task_t){left, task.begin, mid, task.depth + 1};
    }
    free(tasks);
    free(centroid);
    *out_nodes = nodes;
    return node_count;
}

/* detail::build_meshes (src/mesh_build.cpp:91-157): every mesh's tree, concatenated, triangles in leaf order as
 * (v0, e1, e2) float4s, attributes when any mesh has normals. */
static void build_meshes(orc_scene *s, const ngb_mesh *meshes, int mesh_count) {
    int any_attr = 0;
    size_t total_tris = 0, node_cap = 0;
    for (int m = 0; m < mesh_count; ++m) {
        any_attr |= meshes[m].normals != NULL;
        total_tris += (size_t)meshes[m].index_count / 3;
        node_cap += 2 * ((size_t)meshes[m].index_count / 3);
    }
    s->mesh_count = mesh_count;
    s->blas = malloc(sizeof(bnode_t) * (node_cap + 1));
    s->tris = malloc(sizeof(float) * 12 * (total_tris + 1));
    s->tri_index = malloc(sizeof(int32_t) * (total_tris + 1));
    s->attrs = any_attr ? calloc(16 * (total_tris + 1), sizeof(float)) : NULL;
    s->mesh_root = malloc(sizeof(int32_t) * (mesh_count + 1));
    s->mesh_bounds = malloc(sizeof(float) * 6 * (mesh_count + 1));
    s->blas_count = 0;
    s->tri_count = 0;
    for (int m = 0; m < mesh_count; ++m) {
        const ngb_mesh *mesh = &meshes[m];
        const uint32_t tc = (uint32_t)mesh->index_count / 3;
        aabb_t *tb = malloc(sizeof(aabb_t) * (tc + 1));
        for (uint32_t t = 0; t < tc; ++t) {
            aabb_t b = empty_aabb();
            for (int k = 0; k < 3; ++k) {
                const float *v = mesh->vertices + 3 * (size_t)mesh->indices[3 * t + k];
                /* std::fmin / std::fmax as the reference's build compiles them: of two equal values (-0 and
                 * +0) the second, the vertex; glibc's fminf keeps the first (mesh_build.cpp:98-110). */
                for (int a = 0; a < 3; ++a) {
                    b.lo[a] = b.lo[a] < v[a] ? b.lo[a] : v[a];
                    b.hi[a] = b.hi[a] > v[a] ? b.hi[a] : v[a];
                }
            }
            tb[t] = b;
        }
        uint32_t *order = malloc(sizeof(uint32_t) * (tc + 1));
        bnode_t *nodes = NULL;
        const int nn = bvh_build(tb, tc, 4, &nodes, order);
        if (nn <= 0) {
            free(order);
            free(tb);
            continue;
        }
        const int node_base = s->blas_count, tri_base = s->tri_count;
        s->mesh_root[m] = node_base;
        for (int k = 0; k < 3; ++k) {
            s->mesh_bounds[6 * m + k] = nodes[0].lo[k];
            s->mesh_bounds[6 * m + 3 + k] = nodes[0].hi[k];
        }
        for (int i = 0; i < nn; ++i) {
            bnode_t nd = nodes[i];
            nd.a += nd.count > 0 ? tri_base : node_base;
            s->blas[s->blas_count++] = nd;
        }
        for (uint32_t j = 0; j < tc; ++j) {
            const uint32_t t = order[j];
            const float *a = mesh->vertices + 3 * (size_t)mesh->indices[3 * t];
            const float *b = mesh->vertices + 3 * (size_t)mesh->indices[3 * t + 1];
            const float *c = mesh->vertices + 3 * (size_t)mesh->indices[3 * t + 2];
            float *o = s->tris + 12 * (size_t)s->tri_count;
            const float packed[12] = {a[0], a[1], a[2], 0.0f, b[0] - a[0], b[1] - a[1], b[2] - a[2], 0.0f,
                c[0] - a[0], c[1] - a[1], c[2] - a[2], 0.0f};
            memcpy(o, packed, sizeof(packed));
            s->tri_index[s->tri_count] = (int32_t)t;
            if (any_attr) {
                float *rec = s->attrs + 16 * (size_t)s->tri_count;
                const int has_n = mesh->normals != NULL;
                for (int k = 0; k < 3; ++k) {
                    const uint32_t vi = mesh->indices[3 * t + k];
                    if (has_n) {
                        rec[4 * k] = mesh->normals[3 * vi];
                        rec[4 * k + 1] = mesh->normals[3 * vi + 1];
                        rec[4 * k + 2] = mesh->normals[3 * vi + 2];
                    }
                }
                const int32_t flags = has_n ? 1 : 0; /* ATTR_NORMALS (mesh_build.h:28) */
                memcpy(&rec[15], &flags, sizeof(flags));
            }
            s->tri_count++;
        }
        free(nodes);
        free(order);
        free(tb);
    }
}

/* ---------------------------------------------------------------------------------------- compose -- */

/* quat_matrix (src/cuda_backend.cu:165-172), single precision. */
static void quat_matrix(const float *q, float *r) {
    float x = q[0], y = q[1], z = q[2], w = q[3];
    const float n = sqrtf(x * x + y * y + z * z + w * w);
    if (n > 0.0f) {
        x /= n;
        y /= n;
        z /= n;
        w /= n;
    } else {
        x = y = z = 0.0f;
        w = 1.0f;
    }
    r[0] = 1 - 2 * (y * y + z * z);
    r[1] = 2 * (x * y - z * w);
    r[2] = 2 * (x * z + y * w);
    r[3] = 2 * (x * y + z * w);
    r[4] = 1 - 2 * (x * x + z * z);
    r[5] = 2 * (y * z - x * w);
    r[6] = 2 * (x * z - y * w);
    r[7] = 2 * (y * z + x * w);
    r[8] = 1 - 2 * (x * x + y * y);
}

/* bodies_to_matrices (src/cuda_backend.cu:176-202). */
void orc_compose(int worlds, int per_world, int bpw, const int32_t *boi, const float *local_pose, const float *scale,
    const float *poses, float *matrices) {
    const long total = (long)worlds * per_world;
    for (long g = 0; g < total; ++g) {
        const long w = g / per_world, i = g % per_world;
        const float *lp = local_pose + 7 * i, *sc = scale + 3 * i;
        float rl[9], r[9], p[3] = {lp[0], lp[1], lp[2]};
        quat_matrix(lp + 3, rl);
        const int body = boi[i];
        if (body < 0) {
            for (int k = 0; k < 9; ++k) r[k] = rl[k];
        } else {
            const float *bp = poses + 7 * (w * bpw + body);
            float rb[9];
            quat_matrix(bp + 3, rb);
            for (int row = 0; row < 3; ++row) {
                for (int col = 0; col < 3; ++col)
                    r[3 * row + col] = rb[3 * row] * rl[col] + rb[3 * row + 1] * rl[3 + col] + rb[3 * row + 2] * rl[6 + col];
                p[row] = bp[row] + rb[3 * row] * lp[0] + rb[3 * row + 1] * lp[1] + rb[3 * row + 2] * lp[2];
            }
        }
        float *m = matrices + 12 * g;
        for (int row = 0; row < 3; ++row) {
            for (int col = 0; col < 3; ++col) m[4 * row + col] = r[3 * row + col] * sc[col];
            m[4 * row + 3] = p[row];
        }
    }
}

/* ------------------------------------------------------------------------------------------- LBVH -- */
/* src/cuda_tlas.cuh:27-211. */

static inline int32_t f2i(float f) {
    int32_t i;
    memcpy(&i, &f, 4);
    return i;
}
static inline float i2f(int32_t i) {
    float f;
    memcpy(&f, &i, 4);
    return f;
}
static inline int32_t to_ordered(float f) { /* cuda_tlas.cuh:27-30 */
    const int32_t i = f2i(f);
    return i ^ ((i >> 31) & 0x7fffffff);
}
static inline float from_ordered(int32_t i) { return i2f(i ^ ((i >> 31) & 0x7fffffff)); } /* :31 */

/* invert_affine, the device version (cuda_tlas.cuh:35-47): no singularity check. */
static void invert_affine_dev(const float *m, float *out) {
    const float c00 = m[5] * m[10] - m[6] * m[9];
    const float c01 = m[6] * m[8] - m[4] * m[10];
    const float c02 = m[4] * m[9] - m[5] * m[8];
    const float inv = 1.0f / (m[0] * c00 + m[1] * c01 + m[2] * c02);
    const float r[9] = {c00 * inv, (m[2] * m[9] - m[1] * m[10]) * inv, (m[1] * m[6] - m[2] * m[5]) * inv, c01 * inv,
        (m[0] * m[10] - m[2] * m[8]) * inv, (m[2] * m[4] - m[0] * m[6]) * inv, c02 * inv,
        (m[1] * m[8] - m[0] * m[9]) * inv, (m[0] * m[5] - m[1] * m[4]) * inv};
    for (int row = 0; row < 3; ++row) {
        for (int col = 0; col < 3; ++col) out[4 * row + col] = r[3 * row + col];
        out[4 * row + 3] = -(r[3 * row] * m[3] + r[3 * row + 1] * m[7] + r[3 * row + 2] * m[11]);
    }
}

static inline uint32_t spread_bits(uint32_t v) { /* cuda_tlas.cuh:50-56 */
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

static inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

/* common_prefix (cuda_tlas.cuh:119-124). */
static inline int common_prefix(const uint64_t *keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + clz32((uint32_t)(i ^ j));
    return clz64(a ^ b);
}

static int cmp_pair(const void *pa, const void *pb) {
    const uint64_t *a = pa, *b = pb;
    if (a[0] != b[0]) return a[0] < b[0] ? -1 : 1;
    return a[1] < b[1] ? -1 : (a[1] > b[1] ? 1 : 0);
}

/* tlas::Builder::build (cuda_tlas.cuh:266-283) from s->matrices. */
static void build_tlas(orc_scene *s) {
    const int n = s->n, W = s->worlds, P = s->P;
    if (n <= 0 || W <= 0 || P <= 0) return;
    int32_t *wb = malloc(sizeof(int32_t) * 6 * W);
    for (int w = 0; w < W; ++w) /* init_world_bounds (:59-66) */
        for (int k = 0; k < 3; ++k) {
            wb[6 * w + k] = to_ordered(1e30f);
            wb[6 * w + 3 + k] = to_ordered(-1e30f);
        }
    for (int g = 0; g < n; ++g) { /* place_instances (:69-96) */
        const float *m = s->matrices + 12 * (size_t)g;
        invert_affine_dev(m, s->inst[g].inv);
        s->inst[g].blas_root = s->mesh_root[s->slot_mesh[g % P]];
        const float *lb = s->mesh_bounds + 6 * s->slot_mesh[g % P];
        float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
        for (int corner = 0; corner < 8; ++corner) {
            const float p[3] = {(corner & 1) ? lb[3] : lb[0], (corner & 2) ? lb[4] : lb[1], (corner & 4) ? lb[5] : lb[2]};
            for (int a = 0; a < 3; ++a) {
                const float w = m[4 * a] * p[0] + m[4 * a + 1] * p[1] + m[4 * a + 2] * p[2] + m[4 * a + 3];
                lo[a] = fminf(lo[a], w);
                hi[a] = fmaxf(hi[a], w);
            }
        }
        const int world = g / P;
        for (int a = 0; a < 3; ++a) {
            s->aabb[6 * (size_t)g + a] = lo[a];
            s->aabb[6 * (size_t)g + 3 + a] = hi[a];
            const int32_t centre = to_ordered(0.5f * (lo[a] + hi[a]));
            if (centre < wb[6 * world + a]) wb[6 * world + a] = centre;
            if (centre > wb[6 * world + 3 + a]) wb[6 * world + 3 + a] = centre;
        }
    }
    uint64_t *pairs = malloc(sizeof(uint64_t) * 2 * n);
    for (int g = 0; g < n; ++g) { /* make_keys (:99-115) */
        const int world = g / P;
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            const float lo = from_ordered(wb[6 * world + a]), hi = from_ordered(wb[6 * world + 3 + a]);
            const float centre = 0.5f * (s->aabb[6 * (size_t)g + a] + s->aabb[6 * (size_t)g + 3 + a]);
            const float extent = hi - lo;
            const float t = extent > 1e-20f ? (centre - lo) / extent : 0.0f;
            q[a] = (uint32_t)(fminf(fmaxf(t, 0.0f), 1.0f) * 1023.0f);
        }
        const uint32_t morton = (spread_bits(q[0]) << 2) | (spread_bits(q[1]) << 1) | spread_bits(q[2]);
        s->keys[g] = ((uint64_t)world << 32) | morton;
        pairs[2 * g] = s->keys[g];
        pairs[2 * g + 1] = (uint64_t)g;
    }
    /* A stable sort of (key, id), ids ascending, is what cub::DeviceRadixSort::SortPairs gives (:273-274). */
    qsort(pairs, n, 2 * sizeof(uint64_t), cmp_pair);
    for (int k = 0; k < n; ++k) {
        s->sorted_keys[k] = pairs[2 * k];
        s->sorted_ids[k] = (int32_t)pairs[2 * k + 1];
    }
    free(pairs);
    const int nodes = 2 * n - 1;
    int32_t *parent = malloc(sizeof(int32_t) * nodes);
    int32_t *rng = malloc(sizeof(int32_t) * 2 * (n > 1 ? n : 1));
    int32_t *arrivals = calloc(n, sizeof(int32_t));
    int32_t *leaf_world = malloc(sizeof(int32_t) * n);
    for (int v = 0; v < nodes; ++v) parent[v] = -1;
    for (int k = 0; k < n; ++k) { /* make_leaves (:162-175) */
        const int id = s->sorted_ids[k];
        tnode_t *leaf = &s->tlas[n - 1 + k];
        for (int a = 0; a < 3; ++a) {
            leaf->lo[a] = s->aabb[6 * (size_t)id + a];
            leaf->hi[a] = s->aabb[6 * (size_t)id + 3 + a];
        }
        leaf->left = ~id;
        leaf->right = -1;
        leaf_world[k] = id / P;
    }
    const uint64_t *keys = s->sorted_keys;
    for (int i = 0; i < n - 1; ++i) { /* build_radix_tree (:128-159) */
        const int d = common_prefix(keys, n, i, i + 1) > common_prefix(keys, n, i, i - 1) ? 1 : -1;
        const int min_prefix = common_prefix(keys, n, i, i - d);
        int max_length = 2;
        while (common_prefix(keys, n, i, i + max_length * d) > min_prefix) max_length *= 2;
        int length = 0;
        for (int t = max_length / 2; t >= 1; t /= 2)
            if (common_prefix(keys, n, i, i + (length + t) * d) > min_prefix) length += t;
        const int j = i + length * d;
        const int node_prefix = common_prefix(keys, n, i, j);
        int sp = 0;
        for (int t = (length + 1) / 2;; t = (t + 1) / 2) {
            if (common_prefix(keys, n, i, i + (sp + t) * d) > node_prefix) sp += t;
            if (t == 1) break;
        }
        const int gamma = i + sp * d + (d < 0 ? d : 0);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const int left = (lo == gamma) ? n - 1 + gamma : gamma;
        const int right = (hi == gamma + 1) ? n - 1 + gamma + 1 : gamma + 1;
        s->tlas[i].left = left;
        s->tlas[i].right = right;
        parent[left] = i;
        parent[right] = i;
        rng[2 * i] = lo;
        rng[2 * i + 1] = hi;
    }
    for (int k = 0; k < n; ++k) { /* fit_boxes (:179-196), one climb after another */
        int node = n - 1 + k;
        for (;;) {
            const int p = parent[node];
            if (p < 0) break;
            if (arrivals[p]++ == 0) break;
            const int l = s->tlas[p].left, r = s->tlas[p].right;
            for (int a = 0; a < 3; ++a) {
                s->tlas[p].lo[a] = fminf(s->tlas[l].lo[a], s->tlas[r].lo[a]);
                s->tlas[p].hi[a] = fmaxf(s->tlas[l].hi[a], s->tlas[r].hi[a]);
            }
            node = p;
        }
    }
    for (int v = 0; v < nodes; ++v) { /* find_roots (:199-211) */
        const int rx = v < n - 1 ? rng[2 * v] : v - (n - 1), ry = v < n - 1 ? rng[2 * v + 1] : v - (n - 1);
        const int world = leaf_world[rx];
        if (leaf_world[ry] != world) continue;
        const int p = parent[v];
        if (p < 0) {
            s->roots[world] = v;
            continue;
        }
        if (leaf_world[rng[2 * p]] != leaf_world[rng[2 * p + 1]]) s->roots[world] = v;
    }
    free(parent);
    free(rng);
    free(arrivals);
    free(leaf_world);
    free(wb);
}

/* --------------------------------------------------------------------------------------- traversal -- */
/* src/mesh_dev.h:19-227. */

#define NO_HIT 1e30f
#define TLAS_STACK 128
#define BLAS_STACK (60 + 4)

static inline f3 safe_inverse(f3 d) { /* mesh_dev.h:58-61 */
    float x = fabsf(d.x) < 1e-12f ? copysignf(1e-12f, d.x) : d.x;
    float y = fabsf(d.y) < 1e-12f ? copysignf(1e-12f, d.y) : d.y;
    float z = fabsf(d.z) < 1e-12f ? copysignf(1e-12f, d.z) : d.z;
    return mk(1.0f / x, 1.0f / y, 1.0f / z);
}

static inline float box_entry(const float *lo, const float *hi, f3 o, f3 inv_d, float tmax) { /* :66-74 */
    const float tx0 = (lo[0] - o.x) * inv_d.x, tx1 = (hi[0] - o.x) * inv_d.x;
    const float ty0 = (lo[1] - o.y) * inv_d.y, ty1 = (hi[1] - o.y) * inv_d.y;
    const float tz0 = (lo[2] - o.z) * inv_d.z, tz1 = (hi[2] - o.z) * inv_d.z;
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    return tn <= tf ? tn : NO_HIT;
}

/* triangle_hit (:80-99). */
static inline int triangle_hit(const float *tris, int i, f3 o, f3 d, float tmax, float *t, float *bu, float *bv) {
    const float *p0 = tris + 12 * (size_t)i;
    const f3 v0 = mk(p0[0], p0[1], p0[2]), e1 = mk(p0[4], p0[5], p0[6]), e2 = mk(p0[8], p0[9], p0[10]);
    const f3 p = cross3(d, e2);
    const float det = dot3(e1, p);
    if (fabsf(det) < 1e-14f) return 0;
    const float inv_det = 1.0f / det;
    const f3 sv = sub3(o, v0);
    const float u = dot3(sv, p) * inv_det;
    if (u < 0.0f || u > 1.0f) return 0;
    const f3 q = cross3(sv, e1);
    const float v = dot3(d, q) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return 0;
    *t = dot3(e2, q) * inv_det;
    *bu = u;
    *bv = v;
    return *t > 0.0f && *t < tmax;
}

enum { Q_CLOSEST = 0, Q_ANY = 1, Q_COLLECT = 2 };

typedef struct {
    int mode;
    float tmax;
    int inst, tri; /* closest: the hit; collect: the hit to ignore */
    float u, v;
    int found;
    int other_inst, other_tri; /* collect: another object / another triangle of inst within tmax */
    double bytes;
} query_t;

/* traverse<false> over a mesh's tree, with mesh_intersect's / mesh_occluded's leaf (:186-200, :215-222).
 * Returns 1 when an any-hit query found its hit. */
static int blas_walk(const orc_scene *s, int root, f3 o, f3 d, int instance, query_t *q) {
    const f3 inv_d = safe_inverse(d);
    const bnode_t *nodes = s->blas;
    q->bytes += 32;
    if (box_entry(nodes[root].lo, nodes[root].hi, o, inv_d, q->tmax) >= NO_HIT) return 0;
    int stack[BLAS_STACK];
    float stack_t[BLAS_STACK];
    int sp = 0, node = root;
    for (;;) {
        const bnode_t *nd = &nodes[node];
        q->bytes += 32;
        int descended = 0;
        if (nd->count > 0) {
            for (int j = nd->a; j < nd->a + nd->count; ++j) {
                float t, bu, bv;
                q->bytes += 48;
                if (triangle_hit(s->tris, j, o, d, q->tmax, &t, &bu, &bv)) {
                    if (q->mode == Q_ANY) return 1;
                    if (q->mode == Q_CLOSEST) {
                        q->tmax = t;
                        q->inst = instance;
                        q->tri = j;
                        q->u = bu;
                        q->v = bv;
                        q->found = 1;
                    } else {
                        if (instance != q->inst) q->other_inst = 1;
                        else if (j != q->tri) q->other_tri = 1;
                    }
                }
            }
        } else {
            const int a = nd->a, right = nd->a + 1;
            q->bytes += 64;
            const float dl = box_entry(nodes[a].lo, nodes[a].hi, o, inv_d, q->tmax);
            const float dr = box_entry(nodes[right].lo, nodes[right].hi, o, inv_d, q->tmax);
            if (dl < NO_HIT || dr < NO_HIT) {
                const int left_first = dl <= dr;
                const int near_node = left_first ? a : right, far_node = left_first ? right : a;
                const float far_t = left_first ? dr : dl;
                if (far_t < NO_HIT) {
                    stack[sp] = far_node;
                    stack_t[sp] = far_t;
                    ++sp;
                }
                node = near_node;
                descended = 1;
            }
        }
        if (descended) continue;
        while (sp > 0 && stack_t[sp - 1] >= q->tmax) --sp;
        if (sp == 0) return 0;
        node = stack[--sp];
    }
}

static inline f3 to_local_point(const inst_t *in, f3 p) { /* :164-167 */
    const float *m = in->inv;
    return mk(dot3(mk(m[0], m[1], m[2]), p) + m[3], dot3(mk(m[4], m[5], m[6]), p) + m[7],
        dot3(mk(m[8], m[9], m[10]), p) + m[11]);
}
static inline f3 to_local_dir(const inst_t *in, f3 d) { /* :169-171 */
    const float *m = in->inv;
    return mk(dot3(mk(m[0], m[1], m[2]), d), dot3(mk(m[4], m[5], m[6]), d), dot3(mk(m[8], m[9], m[10]), d));
}

/* traverse<true> over a world's tree (:113-159) with mesh_intersect / mesh_occluded (:177-227). */
static int tlas_walk(const orc_scene *s, int world, f3 o, f3 d, query_t *q) {
    const f3 inv_d = safe_inverse(d);
    const tnode_t *nodes = s->tlas;
    const int root = s->roots[world];
    q->bytes += 32;
    if (box_entry(nodes[root].lo, nodes[root].hi, o, inv_d, q->tmax) >= NO_HIT) return 0;
    int stack[TLAS_STACK];
    float stack_t[TLAS_STACK];
    int sp = 0, node = root;
    for (;;) {
        const tnode_t *nd = &nodes[node];
        q->bytes += 32;
        int descended = 0;
        if (nd->left < 0) {
            const int id = ~nd->left;
            const inst_t *in = &s->inst[id];
            q->bytes += 48;
            if (blas_walk(s, in->blas_root, to_local_point(in, o), to_local_dir(in, d), id, q)) return 1;
        } else {
            const int a = nd->left, right = nd->right;
            q->bytes += 64;
            const float dl = box_entry(nodes[a].lo, nodes[a].hi, o, inv_d, q->tmax);
            const float dr = box_entry(nodes[right].lo, nodes[right].hi, o, inv_d, q->tmax);
            if (dl < NO_HIT || dr < NO_HIT) {
                const int left_first = dl <= dr;
                const int near_node = left_first ? a : right, far_node = left_first ? right : a;
                const float far_t = left_first ? dr : dl;
                if (far_t < NO_HIT) {
                    stack[sp] = far_node;
                    stack_t[sp] = far_t;
                    ++sp;
                }
                node = near_node;
                descended = 1;
            }
        }
        if (descended) continue;
        while (sp > 0 && stack_t[sp - 1] >= q->tmax) --sp;
        if (sp == 0) return 0;
        node = stack[--sp];
    }
}

/* ------------------------------------------------------------------------------------ render core -- */
/* src/render_core.h. */

#define MAX_DEPTH 4
#define MIN_THROUGHPUT 1e-3f
#define SURFACE_EPS 1e-3f

typedef struct {
    f3 point, normal;
    mat_t material;
    float t;
    int object;
    int instance, triangle; /* extra: the record of a mesh hit (-1 otherwise) */
    float u, v;
} hit_t;

static inline int sphere_hit(const sphere_t *sp, f3 origin, f3 dir, float *t) { /* :65-75 */
    const f3 L = sub3(sp->center, origin);
    const float tca = dot3(L, dir);
    const float r2 = sp->radius * sp->radius;
    const float d2 = dot3(L, L) - tca * tca;
    if (d2 > r2) return 0;
    const float thc = sqrtf(r2 - d2);
    *t = tca - thc;
    if (*t < 0.0f) *t = tca + thc;
    return *t >= 0.0f;
}

static inline int floor_hit(const plane_t *f, f3 origin, f3 dir, float limit, float *out) { /* :91-99 */
    if (!(fabsf(dir.y) > 1e-3f)) return 0;
    const float d = (f->y - origin.y) / dir.y;
    if (!(d > 0.0f && d < limit)) return 0;
    const f3 pt = add3(origin, muls(dir, d));
    if (fabsf(pt.x) < f->hx && pt.z > f->zmin && pt.z < f->zmax) {
        *out = d;
        return 1;
    }
    return 0;
}

/* mesh_surface (mesh_dev.h:238-262), without textures. */
static void mesh_surface(const orc_scene *s, int instance, int triangle, float hu, float hv, f3 dir, f3 *normal) {
    const float *m = s->inst[instance].inv;
    const f3 r0 = mk(m[0], m[1], m[2]), r1 = mk(m[4], m[5], m[6]), r2 = mk(m[8], m[9], m[10]);
    const float *t = s->tris + 12 * (size_t)triangle;
    const f3 nl = cross3(mk(t[4], t[5], t[6]), mk(t[8], t[9], t[10]));
    f3 geometric = normalize3(add3(add3(muls(r0, nl.x), muls(r1, nl.y)), muls(r2, nl.z)));
    if (dot3(geometric, dir) > 0.0f) geometric = neg3(geometric);
    *normal = geometric;
    if (!s->attrs) return;
    const float *a = s->attrs + 16 * (size_t)triangle;
    int32_t flags;
    memcpy(&flags, &a[15], 4);
    const float w0 = 1.0f - hu - hv;
    if (flags & 1) {
        const f3 n = add3(add3(muls(mk(a[0], a[1], a[2]), w0), muls(mk(a[4], a[5], a[6]), hu)), muls(mk(a[8], a[9], a[10]), hv));
        if (dot3(n, n) > 1e-12f) {
            const f3 smooth = normalize3(add3(add3(muls(r0, n.x), muls(r1, n.y)), muls(r2, n.z)));
            *normal = dot3(smooth, geometric) < 0.0f ? neg3(smooth) : smooth;
        }
    }
}

/* scene_intersect (:78-143). */
static int scene_intersect(const orc_scene *s, int world, f3 origin, f3 dir, hit_t *hit, double *bytes) {
    float best = 1e30f;
    int best_sphere = -1;
    for (int i = 0; i < s->nsph; ++i) {
        float t;
        if (sphere_hit(&s->spheres[i], origin, dir, &t) && t < best) {
            best = t;
            best_sphere = i;
        }
    }
    int hit_floor = 0;
    {
        float d;
        if (floor_hit(&s->floor, origin, dir, best, &d)) {
            best = d;
            hit_floor = 1;
        }
    }
    int best_instance = -1, best_triangle = -1;
    float bu = 0.0f, bv = 0.0f;
    if (s->n > 0) {
        query_t q;
        memset(&q, 0, sizeof(q));
        q.mode = Q_CLOSEST;
        q.tmax = best;
        q.inst = -1;
        q.tri = -1;
        tlas_walk(s, world, origin, dir, &q);
        *bytes += q.bytes;
        if (q.found) {
            best = q.tmax;
            best_instance = q.inst;
            best_triangle = q.tri;
            bu = q.u;
            bv = q.v;
            best_sphere = -1;
            hit_floor = 0;
        }
    }
    if (best_sphere < 0 && !hit_floor && best_instance < 0) return 0;
    hit->t = best;
    hit->point = add3(origin, muls(dir, best));
    hit->instance = -1;
    hit->triangle = -1;
    hit->u = hit->v = 0.0f;
    if (best_instance >= 0) {
        mesh_surface(s, best_instance, best_triangle, bu, bv, dir, &hit->normal);
        const int slot = best_instance % s->P;
        hit->material = s->slot_mat[slot];
        hit->material.diffuse_color = mul3(hit->material.diffuse_color, mk(1.0f, 1.0f, 1.0f));
        hit->object = NGB_OBJECT_INSTANCE + (best_instance - world * s->P);
        hit->instance = best_instance;
        hit->triangle = best_triangle;
        hit->u = bu;
        hit->v = bv;
    } else if (hit_floor) {
        hit->object = NGB_OBJECT_FLOOR;
        hit->normal = mk(0.0f, 1.0f, 0.0f);
        hit->material = s->floor.m;
        const int cx = (int)floorf(hit->point.x * s->floor.checker);
        const int cz = (int)floorf(hit->point.z * s->floor.checker);
        const f3 tint = ((cx + cz) & 1) ? mk(1.0f, 1.0f, 1.0f) : mk(1.0f, 0.7f, 0.3f);
        hit->material.diffuse_color = muls(tint, 0.3f);
    } else {
        hit->normal = normalize3(sub3(hit->point, s->spheres[best_sphere].center));
        hit->material = s->spheres[best_sphere].m;
        hit->object = NGB_OBJECT_SPHERE + best_sphere;
    }
    return 1;
}

/* Another object within 1e-6 relative t of the closest hit, or another triangle of the hit instance. */
static int near_tie(const orc_scene *s, int world, f3 origin, f3 dir, const hit_t *h) {
    const float lim = h->t * (1.0f + 1e-6f);
    int flags = 0;
    for (int i = 0; i < s->nsph; ++i) {
        float t;
        if (h->object != NGB_OBJECT_SPHERE + i && sphere_hit(&s->spheres[i], origin, dir, &t) && t <= lim) flags |= 1;
    }
    if (h->object != NGB_OBJECT_FLOOR) {
        float d;
        if (floor_hit(&s->floor, origin, dir, nextafterf(lim, INFINITY), &d)) flags |= 1;
    }
    if (s->n > 0) {
        query_t q;
        memset(&q, 0, sizeof(q));
        q.mode = Q_COLLECT;
        q.tmax = nextafterf(lim, INFINITY);
        q.inst = h->instance;
        q.tri = h->triangle;
        tlas_walk(s, world, origin, dir, &q);
        if (q.other_inst) flags |= 1;
        if (q.other_tri) flags |= 2;
    }
    return flags;
}

/* scene_occluded (:146-161). */
static int scene_occluded(const orc_scene *s, int world, f3 origin, f3 dir, float max_dist, double *bytes) {
    for (int i = 0; i < s->nsph; ++i) {
        float t;
        if (sphere_hit(&s->spheres[i], origin, dir, &t) && t < max_dist) return 1;
    }
    {
        float d;
        if (floor_hit(&s->floor, origin, dir, max_dist, &d)) return 1;
    }
    if (s->n <= 0) return 0;
    query_t q;
    memset(&q, 0, sizeof(q));
    q.mode = Q_ANY;
    q.tmax = max_dist;
    const int r = tlas_walk(s, world, origin, dir, &q);
    *bytes += q.bytes;
    return r;
}

/* light_factor (device_scene.h:98-111). */
static float light_factor(const light_t *l, f3 towards, float d) {
    float f = 1.0f;
    if (l->falloff > 0.0f) {
        const float q = d / l->falloff;
        f = 1.0f / (1.0f + q * q);
    }
    if (l->cos_outer > -1.5f) {
        const float c = -(l->direction.x * towards.x + l->direction.y * towards.y + l->direction.z * towards.z);
        const float t = fminf(fmaxf((c - l->cos_outer) / fmaxf(l->cos_inner - l->cos_outer, 1e-6f), 0.0f), 1.0f);
        f *= t * t * (3.0f - 2.0f * t);
    }
    return f;
}

static inline f3 offset_origin(f3 p, f3 n, f3 dir) { /* :196-198 */
    return add3(p, muls(n, dot3(dir, n) < 0.0f ? -SURFACE_EPS : SURFACE_EPS));
}

static inline f3 sky(const orc_scene *s, f3 dir) { /* :186-190, the gradient */
    const float t = saturate(dot3(dir, s->env_up) * 0.5f + 0.5f);
    return muls(lerp3(s->env_cd, s->env_cu, t), s->env_int);
}

/* trace (:202-245). tie: set when the first hit of the path is a near tie. */
static f3 trace(const orc_scene *s, int world, f3 origin, f3 dir, uint32_t *rng, int *tie, double *bytes, double *rays) {
    f3 radiance = mk(0.0f, 0.0f, 0.0f);
    float throughput = 1.0f;
    for (int depth = 0;; ++depth) {
        hit_t hit;
        int found = 0;
        if (depth <= MAX_DEPTH) {
            *rays += 1;
            found = scene_intersect(s, world, origin, dir, &hit, bytes);
        }
        if (!found) {
            radiance = add3(radiance, muls(sky(s, dir), throughput));
            break;
        }
        if (depth == 0 && tie && (near_tie(s, world, origin, dir, &hit) & 1)) *tie = 1;
        f3 diffuse = mk(0.0f, 0.0f, 0.0f), specular = mk(0.0f, 0.0f, 0.0f);
        for (int i = 0; i < s->nlig; ++i) {
            const light_t *L = &s->lights[i];
            const f3 lp = add3(L->position, muls(random_unit_vector(rng), L->radius)); /* geom_dev.h:150-152 */
            const f3 to_light = sub3(lp, hit.point);
            const float light_distance = sqrtf(dot3(to_light, to_light));
            const f3 light_dir = muls(to_light, 1.0f / light_distance);
            const float strength = L->intensity * light_factor(L, light_dir, light_distance);
            if (strength <= 0.0f) continue;
            *rays += 1;
            if (scene_occluded(s, world, offset_origin(hit.point, hit.normal, light_dir), light_dir, light_distance, bytes))
                continue;
            const f3 lit = muls(L->color, strength);
            diffuse = add3(diffuse, muls(lit, fmaxf(0.0f, dot3(light_dir, hit.normal))));
            specular = add3(specular,
                muls(lit, powf(fmaxf(0.0f, dot3(reflect3(light_dir, hit.normal), dir)), hit.material.exponent)));
        }
        const f3 direct = add3(mul3(hit.material.diffuse_color, muls(diffuse, hit.material.kd)), muls(specular, hit.material.ks));
        radiance = add3(radiance,
            muls(add3(direct, muls(hit.material.diffuse_color, s->ambient * hit.material.kd)), throughput));
        throughput *= hit.material.kr;
        if (throughput < MIN_THROUGHPUT) break;
        dir = reflect3(dir, hit.normal);
        origin = offset_origin(hit.point, hit.normal, dir);
    }
    return radiance;
}

typedef struct {
    f3 position, right, up, forward;
    float fov_scale, aspect;
} camera_t;

static camera_t camera_from_matrix(const float *m, float fov, int width, int height) { /* :264-273 */
    camera_t c;
    c.position = mk(m[3], m[7], m[11]);
    c.right = normalize3(mk(m[0], m[4], m[8]));
    c.up = normalize3(mk(m[1], m[5], m[9]));
    c.forward = normalize3(mk(-m[2], -m[6], -m[10]));
    c.fov_scale = tanf(fov * 0.5f);
    c.aspect = (float)width / (float)height;
    return c;
}

static inline f3 camera_ray(const camera_t *c, float px, float py, int width, int height) { /* device_scene.h:114-119 */
    const float sx = (2.0f * px / (float)width - 1.0f) * c->fov_scale * c->aspect;
    const float sy = -(2.0f * py / (float)height - 1.0f) * c->fov_scale;
    return normalize3(add3(add3(muls(c->right, sx), muls(c->up, sy)), c->forward));
}

static inline float srgb_channel(float v) { /* geom_dev.h:169-172 */
    const float x = saturate(v);
    return x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
}

/* ------------------------------------------------------------------------------------------ public -- */

static void set_err(char *e, int len, const char *msg) {
    if (e && len > 0) snprintf(e, len, "%s", msg);
}

orc_scene *orc_create(const ngb_scene *sc, char *error, int error_len) {
    if (sc->width <= 0 || sc->height <= 0 || sc->world_count < 1 || sc->cameras_per_world < 1) {
        set_err(error, error_len, "bad frame size or counts");
        return NULL;
    }
    orc_scene *s = calloc(1, sizeof(orc_scene));
    s->W = sc->width;
    s->H = sc->height;
    s->worlds = sc->world_count;
    s->cpw = sc->cameras_per_world;
    s->P = sc->instance_count;
    s->n = s->P * s->worlds;
    s->nsph = sc->sphere_count;
    for (int i = 0; i < s->nsph; ++i) {
        s->spheres[i].center = mk(sc->spheres[i].center.x, sc->spheres[i].center.y, sc->spheres[i].center.z);
        s->spheres[i].radius = sc->spheres[i].radius;
        s->spheres[i].m = to_mat(&sc->spheres[i].material);
    }
    s->nlig = sc->light_count;
    for (int i = 0; i < s->nlig; ++i) { /* device_scene.h:265-272 */
        const ngb_light *l = &sc->lights[i];
        light_t *L = &s->lights[i];
        L->position = mk(l->position.x, l->position.y, l->position.z);
        L->intensity = l->intensity;
        L->radius = l->radius;
        L->falloff = l->falloff;
        f3 d = mk(l->direction.x, l->direction.y, l->direction.z);
        const float nn = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        d = nn > 0.0f ? mk(d.x / nn, d.y / nn, d.z / nn) : mk(0.0f, 0.0f, -1.0f);
        L->direction = d;
        const int spot = l->spot_angle > 0.0f;
        L->cos_outer = spot ? cosf(l->spot_angle) : -2.0f;
        L->cos_inner = spot ? cosf(l->spot_angle * (1.0f - l->spot_softness)) : -2.0f;
        L->color = mk(l->color.x, l->color.y, l->color.z);
    }
    s->floor.y = sc->floor.y;
    s->floor.hx = sc->floor.half_extent_x;
    s->floor.zmin = sc->floor.z_min;
    s->floor.zmax = sc->floor.z_max;
    s->floor.checker = sc->floor.checker_scale;
    s->floor.m = to_mat(&sc->floor.material);
    s->env_up = mk(0.0f, 1.0f, 0.0f);
    s->env_cu = mk(0.10f, 0.26f, 0.60f);
    s->env_cd = mk(0.35f, 0.52f, 0.70f);
    s->env_int = 1.0f;
    s->ambient = 0.0f;
    if (s->P > 0) build_meshes(s, sc->meshes, sc->mesh_count);
    const int P = s->P > 0 ? s->P : 1;
    s->slot_mesh = malloc(sizeof(int32_t) * P);
    s->slot_mat = malloc(sizeof(mat_t) * P);
    for (int i = 0; i < s->P; ++i) {
        s->slot_mesh[i] = sc->instances[i].mesh;
        s->slot_mat[i] = to_mat(&sc->instances[i].material);
    }
    const size_t n = s->n > 0 ? (size_t)s->n : 1;
    s->matrices = malloc(sizeof(float) * 12 * n);
    s->inst = malloc(sizeof(inst_t) * n);
    s->aabb = malloc(sizeof(float) * 6 * n);
    s->keys = malloc(sizeof(uint64_t) * n);
    s->sorted_keys = malloc(sizeof(uint64_t) * n);
    s->sorted_ids = malloc(sizeof(int32_t) * n);
    s->tlas = calloc(2 * n, sizeof(tnode_t));
    s->roots = calloc(s->worlds, sizeof(int32_t));
    for (int w = 0; w < s->worlds; ++w)
        for (int i = 0; i < s->P; ++i) memcpy(s->matrices + 12 * ((size_t)w * s->P + i), sc->instances[i].transform, 48);
    build_tlas(s);
    return s;
}

void orc_destroy(orc_scene *s) {
    if (!s) return;
    free(s->blas);
    free(s->tris);
    free(s->attrs);
    free(s->tri_index);
    free(s->mesh_root);
    free(s->mesh_bounds);
    free(s->slot_mesh);
    free(s->slot_mat);
    free(s->matrices);
    free(s->inst);
    free(s->aabb);
    free(s->keys);
    free(s->sorted_keys);
    free(s->sorted_ids);
    free(s->tlas);
    free(s->roots);
    free(s->boi);
    free(s->lpose);
    free(s->lscale);
    free(s);
}

int orc_set_instance_transforms(orc_scene *s, const float *m) {
    if (s->n == 0) return 0;
    memcpy(s->matrices, m, sizeof(float) * 12 * (size_t)s->n);
    build_tlas(s);
    return 0;
}

int orc_bind_bodies(orc_scene *s, int bpw, const int32_t *boi, const float *lp, const float *sc) {
    const int P = s->P > 0 ? s->P : 1;
    free(s->boi);
    free(s->lpose);
    free(s->lscale);
    s->boi = malloc(sizeof(int32_t) * P);
    s->lpose = malloc(sizeof(float) * 7 * P);
    s->lscale = malloc(sizeof(float) * 3 * P);
    memcpy(s->boi, boi, sizeof(int32_t) * s->P);
    memcpy(s->lpose, lp, sizeof(float) * 7 * s->P);
    memcpy(s->lscale, sc, sizeof(float) * 3 * s->P);
    s->bpw = bpw;
    s->bound = 1;
    return 0;
}

int orc_set_body_poses(orc_scene *s, const float *poses) {
    if (!s->bound) return 1;
    if (s->n == 0) return 0;
    orc_compose(s->worlds, s->P, s->bpw, s->boi, s->lpose, s->lscale, poses, s->matrices);
    build_tlas(s);
    return 0;
}

void orc_set_ambient(orc_scene *s, float a) { s->ambient = a; }

void orc_set_environment(orc_scene *s, const ngb_environment *e) {
    /* Only the gradient's up axis, normalised in double (src/environment.cpp:33-38), and its colours matter. */
    double u[3] = {e->up.x, e->up.y, e->up.z};
    const double un = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    s->env_up = mk((float)(u[0] / un), (float)(u[1] / un), (float)(u[2] / un));
    s->env_cu = mk(e->color_up.x, e->color_up.y, e->color_up.z);
    s->env_cd = mk(e->color_down.x, e->color_down.y, e->color_down.z);
    s->env_int = e->intensity;
}

typedef struct {
    orc_scene *s;
    const float *cameras;
    float fov;
    int spp, frame;
    unsigned outputs;
    uint8_t *rgb;
    float *depth, *normal;
    int32_t *ids, *hit_instance, *hit_triangle;
    float *hit_u, *hit_v;
    uint8_t *ties;
    const float *view;   /* a single-view render's camera as given (14 floats), or NULL: the matrices */
    float *accum;        /* the single-view running sums (4 floats per pixel), or NULL */
    uint32_t *argb;      /* the single-view average's 0xAARRGGBB pixels */
    long total;
    atomic_long next;
    double bytes, rays;
    pthread_mutex_t lock;
} render_job_t;

static void render_pixel(render_job_t *j, long pix, double *bytes, double *rays) {
    orc_scene *s = j->s;
    const int W = s->W, H = s->H;
    const int view = (int)(pix / ((long)W * H));
    const int idx = (int)(pix % ((long)W * H));
    const int y = idx / W, x = idx % W, world = view / s->cpw;
    camera_t cam;
    if (j->view) { /* the Camera as given (cuda_backend.cu:651-652 passes it unchanged) */
        const float *c = j->view;
        cam.position = mk(c[0], c[1], c[2]);
        cam.right = mk(c[3], c[4], c[5]);
        cam.up = mk(c[6], c[7], c[8]);
        cam.forward = mk(c[9], c[10], c[11]);
        cam.fov_scale = c[12];
        cam.aspect = c[13];
    } else {
        cam = camera_from_matrix(j->cameras + 12 * (size_t)view, j->fov, W, H);
    }
    uint8_t tie = 0;
    if (j->outputs & NGB_OUTPUT_RGB) { /* render_pixel_rgb8 (:276-283) via sample_pixel (:248-259) */
        uint32_t r = make_rng((uint32_t)(y * W + x), (uint32_t)j->frame);
        f3 sum = mk(0.0f, 0.0f, 0.0f);
        int t = 0;
        for (int sample = 0; sample < j->spp; ++sample) {
            const float jx = rand_float(&r);
            const float jy = rand_float(&r);
            sum = add3(sum, trace(s, world, cam.position, camera_ray(&cam, (float)x + jx, (float)y + jy, W, H), &r,
                                 j->ties ? &t : NULL, bytes, rays));
        }
        sum = muls(sum, 1.0f / (float)j->spp);
        if (j->accum) { /* render_pixel's running average (render_core.h:288-301) */
            float *a = j->accum + 4 * (size_t)pix;
            if (j->frame == 0) {
                a[0] = sum.x, a[1] = sum.y, a[2] = sum.z, a[3] = 1.0f;
            } else {
                a[0] = a[0] + sum.x, a[1] = a[1] + sum.y, a[2] = a[2] + sum.z, a[3] = a[3] + 1.0f;
            }
            sum = muls(mk(a[0], a[1], a[2]), 1.0f / a[3]);
        }
        const f3 c = mk(srgb_channel(sum.x), srgb_channel(sum.y), srgb_channel(sum.z));
        if (j->argb) { /* pack_argb8888 (geom_dev.h:179-184) */
            const uint32_t r8 = (uint32_t)(saturate(c.x) * 255.0f + 0.5f), g8 = (uint32_t)(saturate(c.y) * 255.0f + 0.5f);
            const uint32_t b8 = (uint32_t)(saturate(c.z) * 255.0f + 0.5f);
            j->argb[pix] = 0xFF000000u | (r8 << 16) | (g8 << 8) | b8;
        }
        if (j->rgb) {
            uint8_t *o = j->rgb + 3 * (size_t)pix;
            o[0] = (uint8_t)(saturate(c.x) * 255.0f + 0.5f);
            o[1] = (uint8_t)(saturate(c.y) * 255.0f + 0.5f);
            o[2] = (uint8_t)(saturate(c.z) * 255.0f + 0.5f);
        }
        if (t) tie |= ORC_TIE_RGB_INSTANCE;
    }
    if (j->outputs & (NGB_OUTPUT_DEPTH | NGB_OUTPUT_NORMAL | NGB_OUTPUT_OBJECT_ID)) { /* aov_pixel (:313-327) */
        const f3 dir = camera_ray(&cam, (float)x + 0.5f, (float)y + 0.5f, W, H);
        hit_t hit;
        *rays += 1;
        const int found = scene_intersect(s, world, cam.position, dir, &hit, bytes);
        if ((j->outputs & NGB_OUTPUT_DEPTH) && j->depth) j->depth[pix] = found ? hit.t * dot3(dir, cam.forward) : INFINITY;
        if ((j->outputs & NGB_OUTPUT_NORMAL) && j->normal) {
            const f3 n = found ? hit.normal : mk(0.0f, 0.0f, 0.0f);
            j->normal[3 * pix] = n.x;
            j->normal[3 * pix + 1] = n.y;
            j->normal[3 * pix + 2] = n.z;
        }
        if ((j->outputs & NGB_OUTPUT_OBJECT_ID) && j->ids) j->ids[pix] = found ? hit.object : NGB_OBJECT_NONE;
        if (j->hit_instance) j->hit_instance[pix] = found ? hit.instance : -1;
        if (j->hit_triangle) j->hit_triangle[pix] = (found && hit.triangle >= 0) ? s->tri_index[hit.triangle] : -1;
        if (j->hit_u) j->hit_u[pix] = found ? hit.u : 0.0f;
        if (j->hit_v) j->hit_v[pix] = found ? hit.v : 0.0f;
        if (j->ties && found) {
            const int f = near_tie(s, world, cam.position, dir, &hit);
            if (f & 1) tie |= ORC_TIE_AOV_INSTANCE;
            if (f & 2) tie |= ORC_TIE_AOV_TRIANGLE;
        }
    }
    if (j->ties) j->ties[pix] = tie;
}

static void *render_worker(void *arg) {
    render_job_t *j = arg;
    double bytes = 0, rays = 0;
    for (;;) {
        const long begin = atomic_fetch_add(&j->next, 256);
        if (begin >= j->total) break;
        const long end = begin + 256 < j->total ? begin + 256 : j->total;
        for (long pix = begin; pix < end; ++pix) render_pixel(j, pix, &bytes, &rays);
    }
    pthread_mutex_lock(&j->lock);
    j->bytes += bytes;
    j->rays += rays;
    pthread_mutex_unlock(&j->lock);
    return NULL;
}

static int run_render(render_job_t *jp, int threads);

int orc_render(orc_scene *s, const float *cameras, float fov, int spp, unsigned outputs, int frame, uint8_t *rgb,
    float *depth, float *normal, int32_t *ids, int32_t *hit_instance, int32_t *hit_triangle, float *hit_u,
    float *hit_v, uint8_t *ties, int threads) {
    render_job_t j;
    memset(&j, 0, sizeof(j));
    j.s = s;
    j.cameras = cameras;
    j.fov = fov;
    j.spp = spp;
    j.frame = frame;
    j.outputs = outputs;
    j.rgb = rgb;
    j.depth = depth;
    j.normal = normal;
    j.ids = ids;
    j.hit_instance = hit_instance;
    j.hit_triangle = hit_triangle;
    j.hit_u = hit_u;
    j.hit_v = hit_v;
    j.ties = ties;
    return run_render(&j, threads);
}

/* The single-view Renderer's render / render_frame (renderer.cpp:104-108, 174-182) for a scene of one world
 * and one camera: camera = position, right, up, forward (3 floats each), fov_scale, aspect, used as given;
 * accum (4 floats per pixel) carries the running average between calls, argb receives its pixels. */
int orc_render_view(orc_scene *s, const float *camera, int spp, unsigned outputs, int frame, float *accum,
    uint32_t *argb, uint8_t *rgb, float *depth, float *normal, int32_t *ids, uint8_t *ties, int threads) {
    render_job_t j;
    memset(&j, 0, sizeof(j));
    j.s = s;
    j.view = camera;
    j.spp = spp;
    j.frame = frame;
    j.outputs = outputs;
    j.rgb = rgb;
    j.depth = depth;
    j.normal = normal;
    j.ids = ids;
    j.ties = ties;
    j.accum = accum;
    j.argb = argb;
    return run_render(&j, threads);
}

static int run_render(render_job_t *jp, int threads) {
    render_job_t j = *jp;
    orc_scene *s = j.s;
    j.total = (long)s->worlds * s->cpw * s->H * s->W;
    atomic_init(&j.next, 0);
    pthread_mutex_init(&j.lock, NULL);
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t pool[256];
    for (int i = 1; i < threads; ++i) pthread_create(&pool[i], NULL, render_worker, &j);
    render_worker(&j);
    for (int i = 1; i < threads; ++i) pthread_join(pool[i], NULL);
    pthread_mutex_destroy(&j.lock);
    s->trav_bytes = j.bytes;
    s->trav_rays = j.rays;
    return 0;
}

int orc_cast_rays(orc_scene *s, const float *origins, const float *directions, int rays_per_world, float max_distance,
    float *distance, float *normal, int32_t *ids) {
    const long count = (long)rays_per_world * s->worlds;
    double bytes = 0;
    for (long i = 0; i < count; ++i) { /* cast_ray (:331-349) */
        const int world = (int)(i / rays_per_world);
        const f3 o = mk(origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]);
        f3 d = mk(directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]);
        const float len2 = dot3(d, d);
        hit_t hit;
        int found = len2 > 1e-30f && len2 < 1e30f;
        if (found) {
            d = muls(d, 1.0f / sqrtf(len2));
            found = scene_intersect(s, world, o, d, &hit, &bytes) && hit.t <= max_distance;
        }
        distance[i] = found ? hit.t : INFINITY;
        const f3 n = found ? hit.normal : mk(0.0f, 0.0f, 0.0f);
        normal[3 * i] = n.x;
        normal[3 * i + 1] = n.y;
        normal[3 * i + 2] = n.z;
        ids[i] = found ? hit.object : NGB_OBJECT_NONE;
    }
    return 0;
}

int orc_tlas(const orc_scene *s, uint64_t *keys, int32_t *sorted_ids, int32_t *nodes, int32_t *roots, float *matrices) {
    const size_t n = (size_t)s->n;
    if (keys) memcpy(keys, s->keys, n * sizeof(uint64_t));
    if (sorted_ids) memcpy(sorted_ids, s->sorted_ids, n * sizeof(int32_t));
    if (nodes && n) memcpy(nodes, s->tlas, (2 * n - 1) * sizeof(tnode_t));
    if (roots) memcpy(roots, s->roots, (size_t)s->worlds * sizeof(int32_t));
    if (matrices) memcpy(matrices, s->matrices, n * 12 * sizeof(float));
    return 0;
}

void orc_blas(const orc_scene *s, int *node_count, int *triangle_count, int32_t *nodes, float *triangles,
    int32_t *roots, float *bounds, int32_t *triangle_index) {
    *node_count = s->blas_count;
    *triangle_count = s->tri_count;
    if (nodes) memcpy(nodes, s->blas, sizeof(bnode_t) * s->blas_count);
    if (triangles) memcpy(triangles, s->tris, sizeof(float) * 12 * s->tri_count);
    if (roots) memcpy(roots, s->mesh_root, sizeof(int32_t) * s->mesh_count);
    if (bounds) memcpy(bounds, s->mesh_bounds, sizeof(float) * 6 * s->mesh_count);
    if (triangle_index) memcpy(triangle_index, s->tri_index, sizeof(int32_t) * s->tri_count);
}

/* The sRGB byte of every float in [0, 1], scanned in order: returns the number of places where the byte goes
 * down (0 when the mapping is monotonic) and fills first[k], the first float whose byte is k or more. */
long long orc_srgb_scan(float *first) {
    long long drops = 0;
    int prev = 0;
    for (int k = 0; k < 256; ++k) first[k] = 2.0f;
    first[0] = 0.0f;
    for (uint32_t bitsv = 0; bitsv <= 0x3f800000u; ++bitsv) {
        float v;
        memcpy(&v, &bitsv, 4);
        const float c = srgb_channel(v);
        const int b = (uint8_t)(saturate(c) * 255.0f + 0.5f);
        if (b < prev) ++drops;
        for (int k = prev + 1; k <= b; ++k) first[k] = v;
        if (b > prev) prev = b;
    }
    return drops;
}

void orc_traversal_bytes(const orc_scene *s, double *bytes, double *rays) {
    *bytes = s->trav_bytes;
    *rays = s->trav_rays;
}
