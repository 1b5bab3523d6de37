// Pose compose and the per-world top-level tree build, fused into one launch.
//
// The tree is the reference's GPU LBVH (src/cuda_tlas.cuh:27-211) node for node: keys world << 32 | Morton
// code of the instance's box centre inside its world's centre bounds, a stable sort, the Karras radix tree
// over all worlds' sorted keys (ties broken by global position), boxes filled bottom-up, and each world's
// root. The reference runs that as ten launches over global memory plus a CUB radix sort. Here, because
// the world sits in the key's top bits, the sorted array is every world's own sorted run laid end to end,
// and every node of a world's subtree depends only on that world's keys and on world numbers. So one group
// of threads per world (a warp, or a whole CTA for up to 1024 instances) does the whole build in shared
// memory: compose the matrix, invert it, box it, reduce the world's centre bounds, make the keys, rank-sort
// them, emit the Karras nodes, and refit the boxes bottom-up with shared-memory atomics. The only nodes a
// group cannot finish are the inter-world ones (never traversed: every ray starts at its world's root);
// their links are emitted by the group that owns their index, and a second small launch fits their boxes
// by climbing from the world roots, as fit_boxes does (cuda_tlas.cuh:179-196).
#include "device.cuh"
#include "kernels.h"

namespace ngb {
namespace {

// quat_matrix (src/cuda_backend.cu:165-172): rotation of a quaternion x, y, z, w, normalised first.
__device__ __forceinline__ void quat_matrix(const float *q, float *r) {
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

// An instance's matrix from its geom's position and rotation and its scale, [R * diag(s) | p]: the products
// of MJWarpBatchRenderer's compose kernel (python/neraulgraphics/mujoco.py:291-302).
__device__ __forceinline__ void compose_geom(const BuildArgs &a, long long w, int i, float *m) {
    const long long geom = w * a.geoms_per_world + __ldg(a.geom_of_instance + i);
    const float *p = a.geom_xpos + 3 * geom, *r = a.geom_xmat + 9 * geom, *sc = a.geom_scale + 3 * i;
    const float s[3] = {__ldg(sc), __ldg(sc + 1), __ldg(sc + 2)};
    for (int row = 0; row < 3; ++row) {
        for (int col = 0; col < 3; ++col) m[4 * row + col] = __ldg(r + 3 * row + col) * s[col];
        m[4 * row + 3] = __ldg(p + row);
    }
}

// An instance's matrix from its body's pose, its own offset and its scale (src/cuda_backend.cu:176-202).
__device__ __forceinline__ void compose(const BuildArgs &a, long long w, int i, float *m) {
    if (a.compose == 2) {
        compose_geom(a, w, i, m);
        return;
    }
    const float *lp = a.local_pose + 7 * i, *sc = a.local_scale + 3 * i;
    float lpv[7], scv[3];
    for (int k = 0; k < 7; ++k) lpv[k] = __ldg(lp + k);
    for (int k = 0; k < 3; ++k) scv[k] = __ldg(sc + k);
    float rl[9], r[9], p[3] = {lpv[0], lpv[1], lpv[2]};
    quat_matrix(lpv + 3, rl);
    const int body = __ldg(a.body_of_instance + i);
    if (body < 0) {
        for (int k = 0; k < 9; ++k) r[k] = rl[k];
    } else {
        const float *bpp = a.body_poses + 7 * (w * a.bodies_per_world + body);
        float bp[7];
        for (int k = 0; k < 7; ++k) bp[k] = __ldg(bpp + k);
        float rb[9];
        quat_matrix(bp + 3, rb);
        for (int row = 0; row < 3; ++row) {
            for (int col = 0; col < 3; ++col)
                r[3 * row + col] = rb[3 * row] * rl[col] + rb[3 * row + 1] * rl[3 + col] + rb[3 * row + 2] * rl[6 + col];
            p[row] = bp[row] + rb[3 * row] * lpv[0] + rb[3 * row + 1] * lpv[1] + rb[3 * row + 2] * lpv[2];
        }
    }
    for (int row = 0; row < 3; ++row) {
        for (int col = 0; col < 3; ++col) m[4 * row + col] = r[3 * row + col] * scv[col];
        m[4 * row + 3] = p[row];
    }
}

// invert_affine (src/cuda_tlas.cuh:35-47), IEEE division.
__device__ __forceinline__ void invert_affine(const float *m, float *out) {
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

// Shared memory of one world's group, G threads (G >= instances per world).
template <int G>
struct GroupSmem {
    uint32_t key_in[G];    // Morton code of local instance i
    uint32_t key[G];       // Morton code at sorted position r
    float box[2 * G][6];   // internal node j at j, leaf of sorted position r at G + r
    int child[G][2];       // local ids of internal node j's children
    int parent[2 * G];     // local id of a node's parent, -1 when it is outside the world
    int arrive[G];
    int sorted[G];         // local instance at sorted position r
    int bounds[6];         // ordered-int centre bounds
};

// The reference's common_prefix (cuda_tlas.cuh:119-124) between sorted positions p (in this world) and x,
// from this world's keys in shared memory and, for a position in another world, from the world numbers
// alone: keys of different worlds first differ in the world bits, so their shared prefix is clz32(w ^ wx).
template <int G>
__device__ __forceinline__ int delta(const GroupSmem<G> &sm, int p, long long x, long long n, long long base, int P,
    uint32_t world, uint32_t key_p, const int *world_first, int worlds) {
    if (x < 0 || x >= n) return -1;
    if (x >= base && x < base + P) {
        const uint32_t kx = sm.key[x - base];
        if (kx == key_p) return 64 + __clz(static_cast<int>(static_cast<uint32_t>(p) ^ static_cast<uint32_t>(x)));
        return 32 + __clz(static_cast<int>(key_p ^ kx));
    }
    uint32_t wx;
    if (world_first) {  // uneven worlds: the last world whose first instance is at most x
        int lo = 0, hi = worlds - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(world_first + mid) <= x) lo = mid;
            else hi = mid - 1;
        }
        wx = static_cast<uint32_t>(lo);
    } else {
        wx = static_cast<uint32_t>(x / P);
    }
    return __clz(static_cast<int>(world ^ wx));
}

template <int G>
__global__ void __launch_bounds__(G < 128 ? 128 : G) build_worlds_kernel(const BuildArgs a) {
    constexpr int CTA = G < 128 ? 128 : G;
    constexpr int WPC = CTA / G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int grp = threadIdx.x / G, i = threadIdx.x % G;
    GroupSmem<G> &sm = reinterpret_cast<GroupSmem<G> *>(smem_raw)[grp];
    const long long w = static_cast<long long>(blockIdx.x) * WPC + grp;
    const long long n = a.n;
    const bool world_ok = w < a.worlds;
    // This world's instances: [base, base + P) (worlds of uneven sizes: from world_first).
    const int P = !world_ok ? 0 : a.world_first ? __ldg(a.world_first + w + 1) - __ldg(a.world_first + w) : a.per_world;
    const bool valid = world_ok && i < P;
    const long long base = !world_ok ? 0 : a.world_first ? __ldg(a.world_first + w) : w * a.per_world;
    const long long g = base + i;
    const int slot = a.world_first ? static_cast<int>(g) : i;  // the slot tables' entry of this instance

    for (int k = i; k < 2 * G; k += G) sm.parent[k] = -1;
    sm.arrive[i] = 0;
    if (i == 0)
        for (int k = 0; k < 3; ++k) {
            sm.bounds[k] = to_ordered(1e30f);
            sm.bounds[3 + k] = to_ordered(-1e30f);
        }
    __syncthreads();

    // Matrix, inverse, world box (place_instances, cuda_tlas.cuh:69-96).
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    if (valid) {
        float m[12];
        if (a.compose) {
            compose(a, w, i, m);
            float *mo = a.matrices_out + 12 * g;
            for (int k = 0; k < 12; ++k) mo[k] = m[k];
        } else {
            const float *mi = a.matrices_in + 12 * g;
            for (int k = 0; k < 12; ++k) m[k] = __ldg(mi + k);
            if (a.matrices_out) {  // matrices in the caller's memory: kept for inspection
                float *mo = a.matrices_out + 12 * g;
                for (int k = 0; k < 12; ++k) mo[k] = m[k];
            }
        }
        float inv[12];
        invert_affine(m, inv);
        float4 *rec = a.inst + 4 * g;
        rec[0] = make_float4(inv[0], inv[1], inv[2], inv[3]);
        rec[1] = make_float4(inv[4], inv[5], inv[6], inv[7]);
        rec[2] = make_float4(inv[8], inv[9], inv[10], inv[11]);
        rec[3] = make_float4(__int_as_float(__ldg(a.slot_blas_root + slot)), __int_as_float(slot), 0.0f, 0.0f);
        const float *lb = a.slot_bounds + 6 * slot;
        float b[6];
        for (int k = 0; k < 6; ++k) b[k] = __ldg(lb + k);
        for (int corner = 0; corner < 8; ++corner) {
            const float p[3] = {(corner & 1) ? b[3] : b[0], (corner & 2) ? b[4] : b[1], (corner & 4) ? b[5] : b[2]};
            for (int ax = 0; ax < 3; ++ax) {
                const float v = m[4 * ax] * p[0] + m[4 * ax + 1] * p[1] + m[4 * ax + 2] * p[2] + m[4 * ax + 3];
                lo[ax] = fminf(lo[ax], v);
                hi[ax] = fmaxf(hi[ax], v);
            }
        }
        for (int ax = 0; ax < 3; ++ax) {
            const int c = to_ordered(0.5f * (lo[ax] + hi[ax]));
            atomicMin(&sm.bounds[ax], c);
            atomicMax(&sm.bounds[3 + ax], c);
        }
    }
    if (world_ok && P == 0 && i == 0) a.roots[w] = -1;  // a world without instances has no tree
    __syncthreads();

    // Key (make_keys, cuda_tlas.cuh:99-115).
    uint32_t morton = 0;
    if (valid) {
        uint32_t q[3];
        for (int ax = 0; ax < 3; ++ax) {
            const float blo = from_ordered(sm.bounds[ax]), bhi = from_ordered(sm.bounds[3 + ax]);
            const float centre = 0.5f * (lo[ax] + hi[ax]);
            const float extent = bhi - blo;
            const float t = extent > 1e-20f ? (centre - blo) / extent : 0.0f;
            q[ax] = static_cast<uint32_t>(fminf(fmaxf(t, 0.0f), 1.0f) * 1023.0f);
        }
        morton = (spread_bits(q[0]) << 2) | (spread_bits(q[1]) << 1) | spread_bits(q[2]);
        a.keys[g] = (static_cast<unsigned long long>(w) << 32) | morton;
        sm.key_in[i] = morton;
    }
    __syncthreads();

    // Stable sort by rank: the sorted position of (key, i) is the number of (key, j) before it. The same
    // order as cub::DeviceRadixSort::SortPairs over (key, id) with ids ascending (cuda_tlas.cuh:273-274).
    int rank = 0;
    if (valid) {
        for (int j = 0; j < P; ++j) {
            const uint32_t kj = sm.key_in[j];
            rank += (kj < morton) || (kj == morton && j < i);
        }
        sm.key[rank] = morton;
        sm.sorted[rank] = i;
        a.sorted_ids[base + rank] = static_cast<int>(g);
        if (a.leaf_of) a.leaf_of[g] = static_cast<int>(base + rank);
        for (int ax = 0; ax < 3; ++ax) {
            sm.box[G + rank][ax] = lo[ax];
            sm.box[G + rank][3 + ax] = hi[ax];
        }
        // The leaf (make_leaves, cuda_tlas.cuh:162-175).
        float4 *leaf = a.tlas + 2 * (n - 1 + base + rank);
        leaf[0] = make_float4(lo[0], lo[1], lo[2], __int_as_float(~static_cast<int>(g)));
        leaf[1] = make_float4(hi[0], hi[1], hi[2], __int_as_float(-1));
    }
    __syncthreads();

    // The internal node at sorted position p = base + i (build_radix_tree, cuda_tlas.cuh:128-159).
    const long long p = base + i;
    bool within = false, is_root = false;
    int left = 0, right = 0;
    if (valid && p < n - 1) {
        const uint32_t kp = sm.key[i];
        const uint32_t wu = static_cast<uint32_t>(w);
        const int ip = static_cast<int>(p);
        auto dlt = [&](long long x) { return delta<G>(sm, ip, x, n, base, P, wu, kp, a.world_first, a.worlds); };
        const int d = dlt(p + 1) > dlt(p - 1) ? 1 : -1;
        const int min_prefix = dlt(p - d);
        long long max_length = 2;
        while (dlt(p + max_length * d) > min_prefix) max_length *= 2;
        long long length = 0;
        for (long long t = max_length / 2; t >= 1; t /= 2)
            if (dlt(p + (length + t) * d) > min_prefix) length += t;
        const long long j = p + length * d;
        const int node_prefix = dlt(j);
        long long s = 0;
        for (long long t = (length + 1) / 2;; t = (t + 1) / 2) {
            if (dlt(p + (s + t) * d) > node_prefix) s += t;
            if (t == 1) break;
        }
        const long long gamma = p + s * d + (d < 0 ? d : 0);
        const long long rlo = p < j ? p : j, rhi = p < j ? j : p;
        left = static_cast<int>((rlo == gamma) ? n - 1 + gamma : gamma);
        right = static_cast<int>((rhi == gamma + 1) ? n - 1 + gamma + 1 : gamma + 1);
        a.parent[left] = ip;
        a.parent[right] = ip;
        within = rlo >= base && rhi <= base + P - 1;
        if (within) {
            auto local = [&](long long c) { return static_cast<int>(c >= n - 1 ? G + (c - (n - 1) - base) : c - base); };
            const int cl = local(left), cr = local(right);
            sm.child[i][0] = cl;
            sm.child[i][1] = cr;
            sm.parent[cl] = i;
            sm.parent[cr] = i;
            is_root = rlo == base && rhi == base + P - 1;
        } else {
            // An inter-world node: its links now, its box from the climb over worlds.
            float4 *nd = a.tlas + 2 * p;
            reinterpret_cast<float *>(nd)[3] = __int_as_float(left);
            reinterpret_cast<float *>(nd + 1)[3] = __int_as_float(right);
        }
        if (is_root) a.roots[w] = ip;
    }
    if (valid && P == 1) a.roots[w] = static_cast<int>(n - 1 + base);
    __syncthreads();

    // Boxes from the leaves up (fit_boxes, cuda_tlas.cuh:179-196): the second of two arrivals at a node
    // knows both children are done, and climbs on.
    if (valid) {
        int node = G + rank;
        volatile float(*vbox)[6] = sm.box;
        for (int steps = 0;; ++steps) {
            const int par = sm.parent[node];
            if (par < 0) break;
            if (steps > 2 * G) {  // longer than any tree over G leaves: the links are malformed
                *a.error_flag = 3;
                break;
            }
            __threadfence_block();
            if (atomicAdd(&sm.arrive[par], 1) == 0) break;
            __threadfence_block();
            const int cl = sm.child[par][0], cr = sm.child[par][1];
            for (int ax = 0; ax < 3; ++ax) {
                vbox[par][ax] = fminf(vbox[cl][ax], vbox[cr][ax]);
                vbox[par][3 + ax] = fmaxf(vbox[cl][3 + ax], vbox[cr][3 + ax]);
            }
            node = par;
        }
    }
    __syncthreads();

    if (valid && p < n - 1 && within) {
        float4 *nd = a.tlas + 2 * p;
        nd[0] = make_float4(sm.box[i][0], sm.box[i][1], sm.box[i][2], __int_as_float(left));
        nd[1] = make_float4(sm.box[i][3], sm.box[i][4], sm.box[i][5], __int_as_float(right));
        if (a.tlas_pairs) {
            // The same node as a child-pair record: both children's boxes and references, (internal node, 0)
            // or (instance, -1) for a leaf.
            const int cl = sm.child[i][0], cr = sm.child[i][1];
            const int rl = cl >= G ? static_cast<int>(base) + sm.sorted[cl - G] : left;
            const int rr = cr >= G ? static_cast<int>(base) + sm.sorted[cr - G] : right;
            const float *bl = sm.box[cl], *br = sm.box[cr];
            float4 *q = a.tlas_pairs + 4 * p;
            q[0] = make_float4(bl[0], bl[1], bl[2], bl[3]);
            q[1] = make_float4(bl[4], bl[5], br[0], br[1]);
            q[2] = make_float4(br[2], br[3], br[4], br[5]);
            q[3] = make_float4(__int_as_float(rl), __int_as_float(cl >= G ? -1 : 0), __int_as_float(rr),
                __int_as_float(cr >= G ? -1 : 0));
        }
    }
}

// The boxes of the inter-world nodes: one thread per world climbs from its root; the second arrival at a
// node computes its box from its children's and climbs on (fit_boxes, cuda_tlas.cuh:179-196). The
// counters are left at zero for the next build.
__global__ void __launch_bounds__(128) fit_world_links_kernel(const int *roots, const int *parent, int *arrivals,
    float4 *tlas, int worlds, int *error_flag) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= worlds) return;
    int node = roots[w];
    if (node < 0) return;
    // Keys of different worlds differ in their 32 world bits, so the tree over worlds is at most 33 deep.
    for (int steps = 0;; ++steps) {
        const int p = parent[node];
        if (p < 0) return;
        if (steps > 64) {
            *error_flag = 4;
            return;
        }
        __threadfence();
        if (atomicAdd(&arrivals[p], 1) == 0) return;
        __threadfence();
        arrivals[p] = 0;
        const float4 p0 = __ldcg(tlas + 2 * p), p1 = __ldcg(tlas + 2 * p + 1);
        const int l = __float_as_int(p0.w), r = __float_as_int(p1.w);
        const float4 l0 = __ldcg(tlas + 2 * l), l1 = __ldcg(tlas + 2 * l + 1);
        const float4 r0 = __ldcg(tlas + 2 * r), r1 = __ldcg(tlas + 2 * r + 1);
        tlas[2 * p] = make_float4(fminf(l0.x, r0.x), fminf(l0.y, r0.y), fminf(l0.z, r0.z), p0.w);
        tlas[2 * p + 1] = make_float4(fmaxf(l1.x, r1.x), fmaxf(l1.y, r1.y), fmaxf(l1.z, r1.z), p1.w);
        node = p;
    }
}

// ------------------------------------------------------------------------------------------------------
// The global build, for worlds of more than MAX_PER_WORLD instances (one large world of 100,000 instances,
// say): the same tree node for node, built over global memory in the reference's steps (cuda_tlas.cuh:69-211)
// with a stable LSD radix sort of its own in place of CUB's.

// Each world's centre bounds start empty.
__global__ void __launch_bounds__(128) init_bounds_kernel(int *bounds, int worlds) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= worlds) return;
    for (int k = 0; k < 3; ++k) {
        bounds[6 * w + k] = to_ordered(1e30f);
        bounds[6 * w + 3 + k] = to_ordered(-1e30f);
    }
}

// Matrix, inverse, record and world box of each instance, and its world's centre bounds (place_instances,
// cuda_tlas.cuh:69-96): the per-world kernel's first step, one thread per instance.
__global__ void __launch_bounds__(128) place_kernel(const BuildArgs a, float4 *aabb, int *bounds) {
    const long long g0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const bool valid = g0 < a.n;
    const long long g = valid ? g0 : a.n - 1;  // lanes past the end repeat the last instance's bounds
    const long long w = g / a.per_world;
    const int i = static_cast<int>(g % a.per_world);
    float m[12];
    if (a.compose) {
        compose(a, w, i, m);
        if (valid) {
            float *mo = a.matrices_out + 12 * g;
            for (int k = 0; k < 12; ++k) mo[k] = m[k];
        }
    } else {
        const float *mi = a.matrices_in + 12 * g;
        for (int k = 0; k < 12; ++k) m[k] = __ldg(mi + k);
        if (valid && a.matrices_out) {  // matrices in the caller's memory: kept for inspection
            float *mo = a.matrices_out + 12 * g;
            for (int k = 0; k < 12; ++k) mo[k] = m[k];
        }
    }
    float inv[12];
    invert_affine(m, inv);
    if (valid) {
        float4 *rec = a.inst + 4 * g;
        rec[0] = make_float4(inv[0], inv[1], inv[2], inv[3]);
        rec[1] = make_float4(inv[4], inv[5], inv[6], inv[7]);
        rec[2] = make_float4(inv[8], inv[9], inv[10], inv[11]);
        rec[3] = make_float4(__int_as_float(__ldg(a.slot_blas_root + i)), __int_as_float(i), 0.0f, 0.0f);
    }
    const float *lb = a.slot_bounds + 6 * i;
    float b[6], lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (int k = 0; k < 6; ++k) b[k] = __ldg(lb + k);
    for (int corner = 0; corner < 8; ++corner) {
        const float p[3] = {(corner & 1) ? b[3] : b[0], (corner & 2) ? b[4] : b[1], (corner & 4) ? b[5] : b[2]};
        for (int ax = 0; ax < 3; ++ax) {
            const float v = m[4 * ax] * p[0] + m[4 * ax + 1] * p[1] + m[4 * ax + 2] * p[2] + m[4 * ax + 3];
            lo[ax] = fminf(lo[ax], v);
            hi[ax] = fmaxf(hi[ax], v);
        }
    }
    if (valid) {
        aabb[2 * g] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        aabb[2 * g + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
    // The world's centre bounds: a block whose instances all sit in one world (a large world's case) reduces
    // them in shared memory and adds one atomic per bound; else a warp in one world reduces first and adds one
    // atomic per bound; otherwise every lane adds its own. (Same-address atomics serialise: 100,000 instances
    // of one world made 19,000 of them per build with one per warp.)
    const long long first = blockIdx.x * static_cast<long long>(blockDim.x);
    const long long wb = (first < a.n ? first : a.n - 1) / a.per_world;
    if (__syncthreads_and(w == wb)) {
        __shared__ int red[32][6];  // per warp: the three minima, then the three maxima
        const int warp = threadIdx.x >> 5;
        for (int ax = 0; ax < 3; ++ax) {
            const int c = to_ordered(0.5f * (lo[ax] + hi[ax]));
            const int mn = __reduce_min_sync(0xffffffffu, c), mx = __reduce_max_sync(0xffffffffu, c);
            if ((threadIdx.x & 31) == 0) {
                red[warp][ax] = mn;
                red[warp][3 + ax] = mx;
            }
        }
        __syncthreads();
        if (threadIdx.x < 6) {
            const int k = threadIdx.x;
            int v = red[0][k];
            for (int q = 1; q < static_cast<int>(blockDim.x >> 5); ++q) v = k < 3 ? min(v, red[q][k]) : max(v, red[q][k]);
            if (k < 3) atomicMin(&bounds[6 * w + k], v);
            else atomicMax(&bounds[6 * w + k], v);
        }
        return;
    }
    const bool one_world = __all_sync(0xffffffffu, w == __shfl_sync(0xffffffffu, w, 0));
    for (int ax = 0; ax < 3; ++ax) {
        int cmin = to_ordered(0.5f * (lo[ax] + hi[ax])), cmax = cmin;
        if (one_world) {
            cmin = __reduce_min_sync(0xffffffffu, cmin);
            cmax = __reduce_max_sync(0xffffffffu, cmax);
            if ((threadIdx.x & 31) != 0) continue;
        }
        atomicMin(&bounds[6 * w + ax], cmin);
        atomicMax(&bounds[6 * w + 3 + ax], cmax);
    }
}

// Keys (make_keys, cuda_tlas.cuh:99-115): world << 32 | Morton code, and the ids to sort with them.
__global__ void __launch_bounds__(128) keys_kernel(const BuildArgs a, const float4 *aabb, const int *bounds,
    unsigned long long *keys_sort, int *ids_sort) {
    const long long g = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (g >= a.n) return;
    const long long w = g / a.per_world;
    const float4 lo = aabb[2 * g], hi = aabb[2 * g + 1];
    const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
    uint32_t q[3];
    for (int ax = 0; ax < 3; ++ax) {
        const float blo = from_ordered(bounds[6 * w + ax]), bhi = from_ordered(bounds[6 * w + 3 + ax]);
        const float centre = 0.5f * (l[ax] + h[ax]);
        const float extent = bhi - blo;
        const float t = extent > 1e-20f ? (centre - blo) / extent : 0.0f;
        q[ax] = static_cast<uint32_t>(fminf(fmaxf(t, 0.0f), 1.0f) * 1023.0f);
    }
    const uint32_t morton = (spread_bits(q[0]) << 2) | (spread_bits(q[1]) << 1) | spread_bits(q[2]);
    const unsigned long long key = (static_cast<unsigned long long>(w) << 32) | morton;
    a.keys[g] = key;
    keys_sort[g] = key;
    ids_sort[g] = static_cast<int>(g);
}

constexpr int SORT_BLOCK = 1024;   // threads per block of a radix pass
constexpr int SORT_ROUNDS = 2;     // runs of SORT_BLOCK consecutive keys per block, taken in order
constexpr long long SORT_TILE = static_cast<long long>(SORT_BLOCK) * SORT_ROUNDS;  // keys per block
constexpr int RADIX = 256;         // 8-bit digits
constexpr int SCAN_ITEMS = 16;     // consecutive counts per thread in the scan

// Radix pass, step 1: each block's count of each digit, stored digit-major (counts[digit * blocks + block]),
// so that one exclusive scan gives every (digit, block) its first output position.
__global__ void __launch_bounds__(SORT_BLOCK) radix_count_kernel(const unsigned long long *keys, long long n, int shift,
    unsigned *counts, int blocks) {
    __shared__ unsigned hist[RADIX];
    if (threadIdx.x < RADIX) hist[threadIdx.x] = 0;
    __syncthreads();
    const long long start = blockIdx.x * SORT_TILE;
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        const long long i = start + static_cast<long long>(r) * SORT_BLOCK + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & (RADIX - 1)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < RADIX) counts[static_cast<long long>(threadIdx.x) * blocks + blockIdx.x] = hist[threadIdx.x];
}

// Radix pass, step 2: exclusive prefix sum of the counts in place, one block: the block walks the array in
// chunks of 1024 x SCAN_ITEMS, each thread summing its SCAN_ITEMS consecutive counts, the thread sums scanned
// with warp shuffles and a scan of the 32 warp totals (one chunk holds the counts of 1,600 blocks of keys).
__global__ void __launch_bounds__(1024) radix_scan_kernel(unsigned *counts, long long total) {
    __shared__ unsigned warp_sum[32];
    __shared__ unsigned carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < total; base += 1024LL * SCAN_ITEMS) {
        const long long k0 = base + static_cast<long long>(threadIdx.x) * SCAN_ITEMS;
        unsigned v[SCAN_ITEMS], sum = 0;
#pragma unroll
        for (int j = 0; j < SCAN_ITEMS; ++j) {
            v[j] = k0 + j < total ? counts[k0 + j] : 0u;
            sum += v[j];
        }
        unsigned x = sum;  // inclusive scan of the thread sums within the warp
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned t = warp_sum[lane];
            for (int off = 1; off < 32; off <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, t, off);
                if (lane >= off) t += y;
            }
            warp_sum[lane] = t;  // inclusive over the warps
        }
        __syncthreads();
        unsigned run = carry + (warp > 0 ? warp_sum[warp - 1] : 0u) + x - sum;
#pragma unroll
        for (int j = 0; j < SCAN_ITEMS; ++j) {
            if (k0 + j < total) counts[k0 + j] = run;
            run += v[j];
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = run;
        __syncthreads();
    }
}

// Radix pass, step 3: every key to its position, stable: its block's running position for its digit (the
// block's first position, advanced by the digit's keys of the block's earlier rounds), plus the keys of that
// digit before it in the round (in earlier warps, counted in shared memory, and earlier lanes of its own warp,
// from the lanes holding the same digit).
__global__ void __launch_bounds__(SORT_BLOCK) radix_scatter_kernel(const unsigned long long *keys_in, const int *ids_in,
    unsigned long long *keys_out, int *ids_out, long long n, int shift, const unsigned *offsets, int blocks) {
    __shared__ unsigned warp_count[SORT_BLOCK / 32][RADIX];
    __shared__ unsigned next[RADIX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < RADIX) next[threadIdx.x] = offsets[static_cast<long long>(threadIdx.x) * blocks + blockIdx.x];
    const long long start = blockIdx.x * SORT_TILE;
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        for (int k = threadIdx.x; k < (SORT_BLOCK / 32) * RADIX; k += SORT_BLOCK) (&warp_count[0][0])[k] = 0;
        __syncthreads();
        const long long i = start + static_cast<long long>(r) * SORT_BLOCK + threadIdx.x;
        const bool valid = i < n;
        const unsigned long long key = valid ? keys_in[i] : 0ull;
        const int digit = valid ? static_cast<int>((key >> shift) & (RADIX - 1)) : RADIX;
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const unsigned rank_in_warp = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank_in_warp == 0) warp_count[warp][digit] = __popc(peers);
        __syncthreads();
        if (valid) {
            unsigned pos = next[digit] + rank_in_warp;
            for (int w = 0; w < warp; ++w) pos += warp_count[w][digit];
            keys_out[pos] = key;
            ids_out[pos] = ids_in[i];
        }
        __syncthreads();
        if (threadIdx.x < RADIX) {
            unsigned t = 0;
            for (int w = 0; w < SORT_BLOCK / 32; ++w) t += warp_count[w][threadIdx.x];
            next[threadIdx.x] += t;
        }
        __syncthreads();  // the sums are read before the next round clears the counts
    }
}

// The leaves in sorted order (make_leaves, cuda_tlas.cuh:162-175), the sorted ids, and each world of one
// instance's root (its leaf).
__global__ void __launch_bounds__(128) leaves_kernel(const BuildArgs a, const int *ids_sorted, const float4 *aabb) {
    const long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (k >= a.n) return;
    const int g = ids_sorted[k];
    a.sorted_ids[k] = g;
    if (a.leaf_of) a.leaf_of[g] = static_cast<int>(k);
    const float4 lo = aabb[2 * static_cast<long long>(g)], hi = aabb[2 * static_cast<long long>(g) + 1];
    float4 *leaf = a.tlas + 2 * (a.n - 1 + k);
    leaf[0] = make_float4(lo.x, lo.y, lo.z, __int_as_float(~g));
    leaf[1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(-1));
    if (k == 0) a.parent[0] = -1;
    if (a.per_world == 1) a.roots[k] = static_cast<int>(a.n - 1 + k);
}

// The Karras node at sorted position p (build_radix_tree + common_prefix, cuda_tlas.cuh:119-159) over the
// sorted 64-bit keys, equal keys told apart by position; and the root of the world whose run it spans.
__global__ void __launch_bounds__(128) karras_kernel(const BuildArgs a, const unsigned long long *skeys) {
    const long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const long long n = a.n;
    if (p >= n - 1) return;
    const unsigned long long kp = skeys[p];
    auto dlt = [&](long long x) -> int {
        if (x < 0 || x >= n) return -1;
        const unsigned long long kx = skeys[x];
        if (kx == kp) return 64 + __clz(static_cast<int>(static_cast<uint32_t>(p) ^ static_cast<uint32_t>(x)));
        return __clzll(static_cast<long long>(kp ^ kx));
    };
    const int d = dlt(p + 1) > dlt(p - 1) ? 1 : -1;
    const int min_prefix = dlt(p - d);
    long long max_length = 2;
    while (dlt(p + max_length * d) > min_prefix) max_length *= 2;
    long long length = 0;
    for (long long t = max_length / 2; t >= 1; t /= 2)
        if (dlt(p + (length + t) * d) > min_prefix) length += t;
    const long long j = p + length * d;
    const int node_prefix = dlt(j);
    long long s = 0;
    for (long long t = (length + 1) / 2;; t = (t + 1) / 2) {
        if (dlt(p + (s + t) * d) > node_prefix) s += t;
        if (t == 1) break;
    }
    const long long gamma = p + s * d + (d < 0 ? d : 0);
    const long long rlo = p < j ? p : j, rhi = p < j ? j : p;
    const int left = static_cast<int>((rlo == gamma) ? n - 1 + gamma : gamma);
    const int right = static_cast<int>((rhi == gamma + 1) ? n - 1 + gamma + 1 : gamma + 1);
    a.parent[left] = static_cast<int>(p);
    a.parent[right] = static_cast<int>(p);
    float4 *nd = a.tlas + 2 * p;
    reinterpret_cast<float *>(nd)[3] = __int_as_float(left);
    reinterpret_cast<float *>(nd + 1)[3] = __int_as_float(right);
    const long long P = a.per_world;
    if (rlo % P == 0 && rhi == rlo + P - 1) a.roots[rlo / P] = static_cast<int>(p);
}

// Boxes from the leaves up (fit_boxes, cuda_tlas.cuh:179-196): the second arrival at a node knows both
// children are done and climbs on; it also writes the node's child-pair record. Counters are left at zero.
__global__ void __launch_bounds__(128) refit_kernel(const BuildArgs a) {
    const long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    const long long n = a.n;
    if (k >= n) return;
    int node = static_cast<int>(n - 1 + k);
    for (int steps = 0;; ++steps) {
        const int par = a.parent[node];
        if (par < 0) return;
        if (steps > 128) {  // deeper than any tree over 64-bit keys: the links are malformed
            *a.error_flag = 3;
            return;
        }
        __threadfence();
        if (atomicAdd(&a.arrivals[par], 1) == 0) return;
        __threadfence();
        a.arrivals[par] = 0;
        const float4 p0 = __ldcg(a.tlas + 2 * par), p1 = __ldcg(a.tlas + 2 * par + 1);
        const int l = __float_as_int(p0.w), r = __float_as_int(p1.w);
        const float4 l0 = __ldcg(a.tlas + 2 * l), l1 = __ldcg(a.tlas + 2 * l + 1);
        const float4 r0 = __ldcg(a.tlas + 2 * r), r1 = __ldcg(a.tlas + 2 * r + 1);
        a.tlas[2 * par] = make_float4(fminf(l0.x, r0.x), fminf(l0.y, r0.y), fminf(l0.z, r0.z), p0.w);
        a.tlas[2 * par + 1] = make_float4(fmaxf(l1.x, r1.x), fmaxf(l1.y, r1.y), fmaxf(l1.z, r1.z), p1.w);
        if (a.tlas_pairs) {
            const bool leaf_l = l >= n - 1, leaf_r = r >= n - 1;
            float4 *q = a.tlas_pairs + 4 * static_cast<long long>(par);
            q[0] = make_float4(l0.x, l0.y, l0.z, l1.x);
            q[1] = make_float4(l1.y, l1.z, r0.x, r0.y);
            q[2] = make_float4(r0.z, r1.x, r1.y, r1.z);
            q[3] = make_float4(__int_as_float(leaf_l ? ~__float_as_int(l0.w) : l), __int_as_float(leaf_l ? -1 : 0),
                __int_as_float(leaf_r ? ~__float_as_int(r0.w) : r), __int_as_float(leaf_r ? -1 : 0));
        }
        node = par;
    }
}

template <int G>
cudaError_t launch_group(const BuildArgs &a, cudaStream_t stream) {
    constexpr int CTA = G < 128 ? 128 : G;
    constexpr int WPC = CTA / G;
    const size_t smem = sizeof(GroupSmem<G>) * WPC;
    cudaError_t e = cudaFuncSetAttribute(build_worlds_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const long long blocks = (a.worlds + WPC - 1) / WPC;
    build_worlds_kernel<G><<<static_cast<unsigned>(blocks), CTA, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace

int large_sort_blocks(long long n) { return static_cast<int>((n + SORT_TILE - 1) / SORT_TILE); }

cudaError_t launch_build_large(const BuildArgs &a, const LargeBuildScratch &t, cudaStream_t stream) {
    if (a.n == 0) return cudaSuccess;
    const long long n = a.n;
    const unsigned grid = static_cast<unsigned>((n + 127) / 128);
    init_bounds_kernel<<<(a.worlds + 127) / 128, 128, 0, stream>>>(t.bounds, a.worlds);
    place_kernel<<<grid, 128, 0, stream>>>(a, t.aabb, t.bounds);
    keys_kernel<<<grid, 128, 0, stream>>>(a, t.aabb, t.bounds, t.keys_a, t.ids_a);
    // Stable LSD radix sort over the Morton bits (0..29) and the world bits (32 and up) of the keys: the order
    // of cub::DeviceRadixSort::SortPairs over (key, id) with ids ascending (cuda_tlas.cuh:241-243, 273-274).
    int world_bits = 0;
    while ((1LL << world_bits) < a.worlds) ++world_bits;
    int shifts[8], passes = 0;
    for (int sh = 0; sh < 32; sh += 8) shifts[passes++] = sh;
    for (int sh = 32; sh < 32 + world_bits; sh += 8) shifts[passes++] = sh;
    const int blocks = large_sort_blocks(n);
    unsigned long long *kin = t.keys_a, *kout = t.keys_b;
    int *iin = t.ids_a, *iout = t.ids_b;
    for (int pass = 0; pass < passes; ++pass) {
        radix_count_kernel<<<blocks, SORT_BLOCK, 0, stream>>>(kin, n, shifts[pass], t.counts, blocks);
        radix_scan_kernel<<<1, 1024, 0, stream>>>(t.counts, static_cast<long long>(RADIX) * blocks);
        radix_scatter_kernel<<<blocks, SORT_BLOCK, 0, stream>>>(kin, iin, kout, iout, n, shifts[pass], t.counts, blocks);
        unsigned long long *kt = kin;
        kin = kout;
        kout = kt;
        int *it = iin;
        iin = iout;
        iout = it;
    }
    leaves_kernel<<<grid, 128, 0, stream>>>(a, iin, t.aabb);
    if (n > 1) {
        karras_kernel<<<static_cast<unsigned>((n - 1 + 127) / 128), 128, 0, stream>>>(a, kin);
        refit_kernel<<<grid, 128, 0, stream>>>(a);
    }
    return cudaGetLastError();
}

int build_group_size(int per_world) {
    int g = 32;
    while (g < per_world) g *= 2;
    return g;
}

cudaError_t launch_build_worlds(const BuildArgs &a, cudaStream_t stream) {
    if (a.n == 0) return cudaSuccess;
    cudaError_t e;
    switch (build_group_size(a.per_world)) {
    case 32: e = launch_group<32>(a, stream); break;
    case 64: e = launch_group<64>(a, stream); break;
    case 128: e = launch_group<128>(a, stream); break;
    case 256: e = launch_group<256>(a, stream); break;
    case 512: e = launch_group<512>(a, stream); break;
    case 1024: e = launch_group<1024>(a, stream); break;
    default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    if (a.worlds > 1) {
        fit_world_links_kernel<<<(a.worlds + 127) / 128, 128, 0, stream>>>(a.roots, a.parent, a.arrivals, a.tlas,
            a.worlds, a.error_flag);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace ngb
