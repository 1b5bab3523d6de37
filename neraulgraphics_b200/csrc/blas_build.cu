// A mesh's bottom-level tree rebuilt on the device from new vertex positions: the binned surface-area-
// heuristic build of src/bvh.cpp:46-174 (16 bins, leaves of at most 4 triangles, depth at most 60) and the
// packing of src/mesh_build.cpp:91-157, giving the host build's tree node for node, its triangles in the
// same leaf order and the same bits.
//
// The host builds depth first from a stack; here the nodes of one depth are split together, one CTA per
// node, level after level, and the host's node numbering is restored at the end:
//   - a node's box, centroid box and bin boxes are min/max reductions. The host's sequential std::min keeps
//     the first of equal values, which matters only for -0 and +0; every reduction here carries the range
//     position of its value and keeps the smallest position among equal values, so the bits are the host's;
//   - std::partition (libstdc++'s bidirectional form) swaps the k-th element from the left that fails the
//     test with the k-th element from the right that passes it, until the two meet: the same swaps are made
//     here from two prefix counts, in parallel;
//   - the host gives a node's two children the indices 2k + 1 and 2k + 2 when it splits the k-th internal
//     node in depth-first, left-first order. An internal node X is preceded in that order by every internal
//     node that starts (in the leaf order) before X does, and by the internal nodes that start where X starts
//     and lie above it (a chain of left children at consecutive depths), so its rank is a prefix count over
//     the start positions plus its depth below the chain's top, with no walk over the tree.
// Node and tree sizes: a tree over T triangles has at most 2T - 1 nodes, numbered in scratch arrays of
// 2T - 1 in level order. The whole build is one cooperative launch: the CTAs (a CTA per large node, a warp per
// small one) split one depth, meet at a grid-wide barrier, and go on to the next depth, whose nodes the splits
// appended after the depth's last node; then the numbering and the packing, between further barriers.
#include <climits>
#include <cstdint>

#include <cooperative_groups.h>

#include "kernels.h"

namespace ngb {
namespace {

constexpr int BINS = 16;
constexpr int MAX_LEAF = 4;
constexpr int MAX_DEPTH = 60;
constexpr unsigned FULL = 0xffffffffu;
constexpr unsigned long long NONE_MIN = ~0ull, NONE_MAX = 0ull;

// Ordering key of a float for min/max with -0 and +0 as one value (the position decides between them).
__device__ __forceinline__ unsigned long long order_key(float v, unsigned pos, bool is_max) {
    const float w = v == 0.0f ? 0.0f : v;
    const unsigned u = __float_as_uint(w);
    const unsigned k = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return (static_cast<unsigned long long>(k) << 32) | (is_max ? 0xffffffffu - pos : pos);
}

__device__ __forceinline__ unsigned key_pos(unsigned long long key, bool is_max) {
    const unsigned low = static_cast<unsigned>(key);
    return is_max ? 0xffffffffu - low : low;
}

__device__ __forceinline__ unsigned long long shfl_u64(unsigned long long v, int mask) {
    const unsigned lo = __shfl_xor_sync(FULL, static_cast<unsigned>(v), mask);
    const unsigned hi = __shfl_xor_sync(FULL, static_cast<unsigned>(v >> 32), mask);
    return (static_cast<unsigned long long>(hi) << 32) | lo;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
    for (int m = 16; m > 0; m >>= 1) {
        const unsigned long long o = shfl_u64(v, m);
        v = o < v ? o : v;
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
    for (int m = 16; m > 0; m >>= 1) {
        const unsigned long long o = shfl_u64(v, m);
        v = o > v ? o : v;
    }
    return v;
}

// The host's box arithmetic (bvh::grow with std::min / std::max, bvh::surface_area).
struct Box {
    float lo[3], hi[3];
};

__device__ __forceinline__ Box empty_box() {
    const float inf = __int_as_float(0x7f800000);
    return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}

__device__ __forceinline__ void grow(Box &b, const Box &o) {
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = o.lo[k] < b.lo[k] ? o.lo[k] : b.lo[k];
        b.hi[k] = b.hi[k] < o.hi[k] ? o.hi[k] : b.hi[k];
    }
}

__device__ __forceinline__ float area(const Box &b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
    const int b = static_cast<int>((c - lo) * scale);
    return b < BINS - 1 ? b : BINS - 1;
}

// Triangle boxes (the vertices' std::fmin / std::fmax in vertex order, src/mesh_build.cpp, as the host build
// computes them: of two equal values, -0 and +0, the later one) and centroids (0.5 (lo + hi),
// src/bvh.cpp:55-56); the order starts as the identity and the root spans every triangle.
__device__ void prepare_item(const MeshBuildArgs &a, const MeshBuildScratch &t, int i) {
    t.starts[i] = 0;
    t.top[i] = INT_MAX;
    Box b = empty_box();
    for (int k = 0; k < 3; ++k) {
        const float *v = a.vertices + 3 * static_cast<size_t>(__ldg(a.indices + 3 * static_cast<size_t>(i) + k));
        for (int c = 0; c < 3; ++c) {
            const float x = __ldg(v + c);
            b.lo[c] = b.lo[c] < x ? b.lo[c] : x;
            b.hi[c] = b.hi[c] > x ? b.hi[c] : x;
        }
    }
    for (int c = 0; c < 3; ++c) {
        t.box[6 * static_cast<size_t>(i) + c] = b.lo[c];
        t.box[6 * static_cast<size_t>(i) + 3 + c] = b.hi[c];
        t.centre[3 * static_cast<size_t>(i) + c] = 0.5f * (b.lo[c] + b.hi[c]);
    }
    t.order[i] = static_cast<uint32_t>(i);
}

template <int WARPS>
struct SplitSmem {
    unsigned long long box_key[12];              // node box lo/hi (6), centroid box lo/hi (6)
    unsigned long long bin_key[3][BINS][6];      // per axis and bin: its box lo/hi
    int bin_count[3][BINS];
    float node[12];                              // the decoded node box and centroid box
    float bin_box[3][BINS][6];                   // the decoded bin boxes (empty bins: +inf lo, -inf hi)
    int warp_sum[WARPS];
    int total;
    float cbox[6];
    int best_axis, best_bin, leaf, mid;
};

// A barrier over the threads that split one node: the CTA, or one warp.
template <int WARPS>
__device__ __forceinline__ void group_sync() {
    if constexpr (WARPS == 1) __syncwarp();
    else __syncthreads();
}

// Exclusive prefix sum of v over the group's threads (gtid: the thread's place in the group; in thread order,
// or from the last thread down when reverse), and the group's total.
template <int WARPS>
__device__ __forceinline__ int cta_scan(SplitSmem<WARPS> &sm, int v, bool reverse, int &total, int gtid) {
    const int lane = gtid & 31, warp = gtid >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = reverse ? __shfl_down_sync(FULL, incl, o) : __shfl_up_sync(FULL, incl, o);
        if (reverse ? lane + o < 32 : lane >= o) incl += u;
    }
    if (reverse ? lane == 0 : lane == 31) sm.warp_sum[warp] = incl;
    group_sync<WARPS>();
    int before = 0;
    total = 0;
    for (int w = 0; w < WARPS; ++w) {
        before += (reverse ? w > warp : w < warp) ? sm.warp_sum[w] : 0;
        total += sm.warp_sum[w];
    }
    group_sync<WARPS>();
    return before + incl - v;
}

// Splits node x at this depth with a group of THREADS threads (tid: the thread's place in the group): 256 for
// the upper depths' large nodes, one warp for the lower depths' small ones. Its children, if any, take the
// next two places after next_first (the next depth's first node) counted by next_count.
template <int THREADS>
__device__ void split_node(const MeshBuildArgs &a, const MeshBuildScratch &t, int x, int depth, SplitSmem<THREADS / 32> &sm,
    int tid, int next_first, int *next_count) {
    constexpr int WARPS = THREADS / 32;
    const int lane = tid & 31;
    {
        const int begin = t.begin[x], end = t.end[x], count = end - begin;
        if (tid == 0) t.depth[x] = depth;
        for (int k = tid; k < 12; k += THREADS) sm.box_key[k] = (k % 6) < 3 ? NONE_MIN : NONE_MAX;
        for (int k = tid; k < 3 * BINS * 6; k += THREADS)
            (&sm.bin_key[0][0][0])[k] = (k % 6) < 3 ? NONE_MIN : NONE_MAX;
        for (int k = tid; k < 3 * BINS; k += THREADS) (&sm.bin_count[0][0])[k] = 0;
        group_sync<WARPS>();

        // The node's box and centroid box: per thread the first of its smallest / largest values, then the
        // warp's and the CTA's by (value, position).
        {
            float best[12];
            unsigned pos[12];
            for (int k = 0; k < 12; ++k) {
                best[k] = (k % 6) < 3 ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
                pos[k] = 0xffffffffu;
            }
            for (int i = begin + tid; i < end; i += THREADS) {
                const uint32_t p = t.order[i];
                float v[12];
                for (int c = 0; c < 6; ++c) v[c] = t.box[6 * static_cast<size_t>(p) + c];
                for (int c = 0; c < 3; ++c) v[6 + c] = v[9 + c] = t.centre[3 * static_cast<size_t>(p) + c];
                for (int k = 0; k < 12; ++k) {
                    const bool take = (k % 6) < 3 ? v[k] < best[k] : best[k] < v[k];
                    if (take || pos[k] == 0xffffffffu) {
                        best[k] = v[k];
                        pos[k] = static_cast<unsigned>(i);
                    }
                }
            }
            for (int k = 0; k < 12; ++k) {
                const bool is_max = (k % 6) >= 3;
                unsigned long long key = pos[k] == 0xffffffffu ? (is_max ? NONE_MAX : NONE_MIN)
                                                                : order_key(best[k], pos[k], is_max);
                key = is_max ? warp_max_u64(key) : warp_min_u64(key);
                if (lane == 0) {
                    if (is_max) atomicMax(&sm.box_key[k], key);
                    else atomicMin(&sm.box_key[k], key);
                }
            }
        }
        group_sync<WARPS>();
        if (tid < 12) {  // the values the keys point at, one per thread
            const bool is_max = (tid % 6) >= 3;
            const uint32_t p = t.order[key_pos(sm.box_key[tid], is_max)];
            sm.node[tid] = tid < 6 ? t.box[6 * static_cast<size_t>(p) + tid] : t.centre[3 * static_cast<size_t>(p) + (tid - 6) % 3];
        }
        group_sync<WARPS>();
        Box box;
        float cb[6];
        for (int k = 0; k < 3; ++k) {
            box.lo[k] = sm.node[k];
            box.hi[k] = sm.node[3 + k];
        }
        for (int k = 0; k < 6; ++k) cb[k] = sm.node[6 + k];

        // Bins on every axis whose centroids spread (src/bvh.cpp:94-107).
        if (count > 1) {
            for (int i = begin + tid; i < end; i += THREADS) {
                const uint32_t p = t.order[i];
                for (int axis = 0; axis < 3; ++axis) {
                    const float extent = cb[3 + axis] - cb[axis];
                    if (!(extent > 0.0f)) continue;
                    const float scale = static_cast<float>(BINS) / extent;
                    const int b = bin_of(t.centre[3 * static_cast<size_t>(p) + axis], cb[axis], scale);
                    atomicAdd(&sm.bin_count[axis][b], 1);
                    // The shared value only moves one way, so a key that does not beat it now never will:
                    // most keys are dropped by a plain read instead of a contended atomic.
                    for (int c = 0; c < 6; ++c) {
                        const bool is_max = c >= 3;
                        const unsigned long long key = order_key(t.box[6 * static_cast<size_t>(p) + c],
                            static_cast<unsigned>(i), is_max);
                        unsigned long long *slot = &sm.bin_key[axis][b][c];
                        const unsigned long long now = *reinterpret_cast<volatile unsigned long long *>(slot);
                        if (is_max ? key > now : key < now) {
                            if (is_max) atomicMax(slot, key);
                            else atomicMin(slot, key);
                        }
                    }
                }
            }
        }
        group_sync<WARPS>();
        for (int e = tid; e < 3 * BINS * 6; e += THREADS) {  // the bin boxes' values, in parallel
            const int axis = e / (BINS * 6), b = (e / 6) % BINS, c = e % 6;
            float v = c < 3 ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
            if (count > 1 && sm.bin_count[axis][b] > 0) {
                const uint32_t p = t.order[key_pos(sm.bin_key[axis][b][c], c >= 3)];
                v = t.box[6 * static_cast<size_t>(p) + c];
            }
            sm.bin_box[axis][b][c] = v;
        }
        group_sync<WARPS>();

        // The split: the cheapest plane over the axes in order, then the leaf test (src/bvh.cpp:108-146).
        if (tid == 0) {
            int best_axis = -1, best_bin = 0;
            float best_cost = __int_as_float(0x7f800000);
            if (count > 1) {
                for (int axis = 0; axis < 3; ++axis) {
                    const float extent = cb[3 + axis] - cb[axis];
                    if (!(extent > 0.0f)) continue;
                    Box bins[BINS];
                    for (int b = 0; b < BINS; ++b)
                        for (int c = 0; c < 3; ++c) {
                            bins[b].lo[c] = sm.bin_box[axis][b][c];
                            bins[b].hi[c] = sm.bin_box[axis][b][3 + c];
                        }
                    float right_area[BINS - 1];
                    int right_count[BINS - 1];
                    Box acc = empty_box();
                    int running = 0;
                    for (int i = BINS - 1; i >= 1; --i) {
                        grow(acc, bins[i]);
                        running += sm.bin_count[axis][i];
                        right_area[i - 1] = area(acc);
                        right_count[i - 1] = running;
                    }
                    acc = empty_box();
                    running = 0;
                    for (int i = 0; i < BINS - 1; ++i) {
                        grow(acc, bins[i]);
                        running += sm.bin_count[axis][i];
                        if (running == 0 || right_count[i] == 0) continue;
                        const float cost = static_cast<float>(running) * area(acc) +
                            static_cast<float>(right_count[i]) * right_area[i];
                        if (cost < best_cost) {
                            best_cost = cost;
                            best_axis = axis;
                            best_bin = i;
                        }
                    }
                }
            }
            const float leaf_cost = static_cast<float>(count) * area(box);
            const float split_cost = 1.0f * area(box) + best_cost;
            const bool small = count <= MAX_LEAF;
            sm.leaf = (count == 1 || depth >= MAX_DEPTH || (small && (best_axis < 0 || leaf_cost <= split_cost))) ? 1 : 0;
            sm.best_axis = best_axis;
            sm.best_bin = best_bin;
            for (int c = 0; c < 6; ++c) sm.cbox[c] = cb[c];
        }
        group_sync<WARPS>();
        const int leaf = sm.leaf, best_axis = sm.best_axis, best_bin = sm.best_bin;
        if (tid < 6) t.node_box[6 * static_cast<size_t>(x) + tid] = tid < 3 ? box.lo[tid] : box.hi[tid - 3];
        if (leaf) {
            if (tid == 0) t.left[x] = -1;
            group_sync<WARPS>();
            return;
        }

        // std::partition over the range by (bin <= best_bin): the k-th failing element from the left swaps
        // with the k-th passing element from the right, for every k before the two runs meet.
        int mid = begin + count / 2;
        if (best_axis >= 0) {
            const float lo = sm.cbox[best_axis];
            const float scale = static_cast<float>(BINS) / (sm.cbox[3 + best_axis] - lo);
            auto passes = [&](int i) {
                return bin_of(t.centre[3 * static_cast<size_t>(t.order[i]) + best_axis], lo, scale) <= best_bin;
            };
            // Each thread takes a contiguous run of the range: it counts, the CTA scans the counts, and it
            // writes its run's positions in order.
            const int run = (count + THREADS - 1) / THREADS;
            const int r0 = begin + tid * run < end ? begin + tid * run : end;
            const int r1 = r0 + run < end ? r0 + run : end;
            int mine = 0;
            for (int i = r0; i < r1; ++i) mine += passes(i) ? 1 : 0;
            int passing;
            cta_scan(sm, mine, false, passing, tid);
            const int meet = begin + passing;
            // Failing elements left of meet, ranked from the left; passing ones right of it, from the right.
            const int l1 = r1 < meet ? r1 : meet, q0 = r0 > meet ? r0 : meet;
            int fails = 0, passes_right = 0;
            for (int i = r0; i < l1; ++i) fails += passes(i) ? 0 : 1;
            for (int j = q0; j < r1; ++j) passes_right += passes(j) ? 1 : 0;
            int swaps, found;
            const int lbase = cta_scan(sm, fails, false, swaps, tid);
            const int rbase = cta_scan(sm, passes_right, true, found, tid);
            for (int i = r0, k = lbase; i < l1; ++i)
                if (!passes(i)) t.lpos[begin + k++] = i;
            for (int j = r1 - 1, k = rbase; j >= q0; --j)
                if (passes(j)) t.rpos[begin + k++] = j;
            group_sync<WARPS>();
            for (int k = tid; k < swaps; k += THREADS) {
                const int l = t.lpos[begin + k], r = t.rpos[begin + k];
                const uint32_t pl = t.order[l];
                t.order[l] = t.order[r];
                t.order[r] = pl;
            }
            mid = meet;
            if (mid == begin || mid == end) mid = begin + count / 2;
        }
        group_sync<WARPS>();
        if (tid == 0) {
            const int c = next_first + atomicAdd(next_count, 2);
            t.left[x] = c;
            t.begin[c] = begin;
            t.end[c] = mid;
            t.begin[c + 1] = mid;
            t.end[c + 1] = end;
        }
        group_sync<WARPS>();
    }
}

// The packed tree (src/mesh_build.cpp:91-157): bvh::Node records with global indices, and the child-pair
// records of the internal nodes.
__device__ void write_node(const MeshBuildArgs &a, const MeshBuildScratch &t, int x) {
    const int i = t.index[x];
    const float *b = t.node_box + 6 * static_cast<size_t>(x);
    const int l = t.left[x];
    float4 *node = a.blas + 2 * (static_cast<size_t>(a.node_base) + i);
    float4 *pair = a.pairs + 4 * (static_cast<size_t>(a.node_base) + i);
    if (l < 0) {
        node[0] = make_float4(b[0], b[1], b[2], __int_as_float(a.tri_base + t.begin[x]));
        node[1] = make_float4(b[3], b[4], b[5], __int_as_float(t.end[x] - t.begin[x]));
        const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        pair[0] = pair[1] = pair[2] = pair[3] = z;
        return;
    }
    node[0] = make_float4(b[0], b[1], b[2], __int_as_float(a.node_base + t.index[l]));
    node[1] = make_float4(b[3], b[4], b[5], __int_as_float(0));
    const float *lb = t.node_box + 6 * static_cast<size_t>(l), *rb = t.node_box + 6 * static_cast<size_t>(l + 1);
    int ref[4];
    for (int c = 0; c < 2; ++c) {
        const int y = l + c;
        const bool y_leaf = t.left[y] < 0;
        ref[2 * c] = y_leaf ? a.tri_base + t.begin[y] : a.node_base + t.index[y];
        ref[2 * c + 1] = y_leaf ? t.end[y] - t.begin[y] : 0;
    }
    pair[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
    pair[1] = make_float4(lb[4], lb[5], rb[0], rb[1]);
    pair[2] = make_float4(rb[2], rb[3], rb[4], rb[5]);
    pair[3] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]), __int_as_float(ref[3]));
}

// Triangles in leaf order (v0, e1 = v1 - v0, e2 = v2 - v0), their mesh indices both ways, and their vertex
// normals (ATTR_NORMALS, src/mesh_build.h:28) where the scene keeps them.
__device__ void write_triangle(const MeshBuildArgs &a, const MeshBuildScratch &t, int p) {
    const uint32_t tri = t.order[p];
    const size_t packed = static_cast<size_t>(a.tri_base) + p;
    float3 v[3];
    for (int k = 0; k < 3; ++k) {
        const float *q = a.vertices + 3 * static_cast<size_t>(__ldg(a.indices + 3 * static_cast<size_t>(tri) + k));
        v[k] = make_float3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
    }
    a.tris[3 * packed] = make_float4(v[0].x, v[0].y, v[0].z, 0.0f);
    a.tris[3 * packed + 1] = make_float4(v[1].x - v[0].x, v[1].y - v[0].y, v[1].z - v[0].z, 0.0f);
    a.tris[3 * packed + 2] = make_float4(v[2].x - v[0].x, v[2].y - v[0].y, v[2].z - v[0].z, 0.0f);
    a.tri_index[packed] = static_cast<int>(tri);
    a.tri_of_local[static_cast<size_t>(a.tri_base) + tri] = static_cast<int>(packed);
    if (!a.attrs) return;
    float rec[16] = {};
    if (a.normals)
        for (int k = 0; k < 3; ++k) {
            const float *q = a.normals + 3 * static_cast<size_t>(__ldg(a.indices + 3 * static_cast<size_t>(tri) + k));
            rec[4 * k] = __ldg(q);
            rec[4 * k + 1] = __ldg(q + 1);
            rec[4 * k + 2] = __ldg(q + 2);
        }
    rec[15] = __int_as_float(a.normals ? 1 : 0);
    for (int k = 0; k < 4; ++k) a.attrs[4 * packed + k] = make_float4(rec[4 * k], rec[4 * k + 1], rec[4 * k + 2], rec[4 * k + 3]);
}

// The slots of this mesh: their root reference, their box in mesh space, and no convexity claim (the new
// shape is not checked).
__device__ void write_slot(const MeshBuildArgs &a, const MeshBuildScratch &t, const int *slot_mesh, int mesh,
    int2 *slot_root, float *slot_bounds, float4 *slot_hull, int s) {
    if (slot_mesh[s] != mesh) return;
    const bool leaf = t.left[0] < 0;
    slot_root[s] = leaf ? make_int2(a.tri_base, a.triangles) : make_int2(a.node_base, 0);
    for (int c = 0; c < 6; ++c) slot_bounds[6 * static_cast<size_t>(s) + c] = t.node_box[c];
    slot_hull[s].w = -1.0f;
}

// The whole build, one cooperative launch of CTAs of 256 threads; grid-wide barriers between its phases.
__global__ void __launch_bounds__(256) build_mesh_kernel(const MeshBuildArgs a, const MeshBuildScratch t,
    const int *slot_mesh, int slots, int mesh, int2 *slot_root, float *slot_bounds, float4 *slot_hull) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    __shared__ SplitSmem<8> cta_smem;
    __shared__ SplitSmem<1> warp_smem[8];
    __shared__ int prefix_warp[8];
    __shared__ int prefix_carry;
    const long long rank = grid.thread_rank(), size = grid.size();
    const int T = a.triangles;
    const long long cap = 2LL * T - 1;

    // The mesh's whole node run cleared, the triangles' boxes, the root spanning every triangle.
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (long long k = rank; k < 2 * cap; k += size) a.blas[2LL * a.node_base + k] = zero;
    for (long long k = rank; k < 4 * cap; k += size) a.pairs[4LL * a.node_base + k] = zero;
    for (long long i = rank; i < T; i += size) prepare_item(a, t, static_cast<int>(i));
    for (long long d = rank; d <= MESH_LEVELS; d += size) t.level_count[d] = 0;
    if (rank == 0) {
        t.begin[0] = 0;
        t.end[0] = T;
        t.index[0] = 0;
    }
    grid.sync();

    // Depth after depth: the splits of depth d append depth d + 1's nodes after depth d's last.
    int first = 0, last = 1;
    for (int depth = 0; depth < MESH_LEVELS && first < last; ++depth) {
        int *next_count = t.level_count + depth + 1;
        if ((static_cast<long long>(T) >> depth) > 512) {
            for (int x = first + blockIdx.x; x < last; x += gridDim.x)
                split_node<256>(a, t, x, depth, cta_smem, threadIdx.x, last, next_count);
        } else {
            const int w = threadIdx.x >> 5;
            for (int x = first + blockIdx.x * 8 + w; x < last; x += gridDim.x * 8)
                split_node<32>(a, t, x, depth, warp_smem[w], threadIdx.x & 31, last, next_count);
        }
        grid.sync();
        const int next = last + __ldcg(next_count);
        first = last;
        last = next;
    }
    const int nodes = last;

    // Per start position: the internal nodes starting there and the least depth among them; their prefix sum
    // (one CTA); then the host's node indices: the k-th internal node in depth-first order has children 2k + 1
    // and 2k + 2.
    for (long long x = rank; x < nodes; x += size)
        if (t.left[x] >= 0) {
            atomicAdd(t.starts + t.begin[x], 1);
            atomicMin(t.top + t.begin[x], t.depth[x]);
        }
    grid.sync();
    if (blockIdx.x == 0) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (threadIdx.x == 0) prefix_carry = 0;
        __syncthreads();
        for (int base = 0; base < T; base += 256) {
            const int i = base + threadIdx.x;
            const int v = i < T ? __ldcg(t.starts + i) : 0;
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += u;
            }
            if (lane == 31) prefix_warp[warp] = incl;
            __syncthreads();
            int before = prefix_carry;
            for (int k = 0; k < warp; ++k) before += prefix_warp[k];
            if (i < T) t.prefix[i] = before + incl - v;
            __syncthreads();
            if (threadIdx.x == 255) prefix_carry = before + incl;
            __syncthreads();
        }
    }
    grid.sync();
    for (long long x = rank; x < nodes; x += size) {
        const int l = t.left[x];
        if (l < 0) continue;
        const int b = t.begin[x];
        const int k = t.prefix[b] + t.depth[x] - __ldcg(t.top + b);
        t.index[l] = 2 * k + 1;
        t.index[l + 1] = 2 * k + 2;
    }
    if (rank == 0) *t.counter = nodes;
    grid.sync();

    // The packed tree, its triangles, and the slots of this mesh.
    for (long long x = rank; x < nodes; x += size) write_node(a, t, static_cast<int>(x));
    for (long long p = rank; p < T; p += size) write_triangle(a, t, static_cast<int>(p));
    for (long long k = rank; k < slots; k += size)
        write_slot(a, t, slot_mesh, mesh, slot_root, slot_bounds, slot_hull, static_cast<int>(k));
}

}  // namespace

cudaError_t launch_mesh_build(const MeshBuildArgs &a, const MeshBuildScratch &t, const int *slot_mesh, int slots,
    int mesh, int2 *slot_root, float *slot_bounds, float4 *slot_hull, cudaStream_t stream) {
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, build_mesh_kernel, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    // Every CTA resident at once (the barriers need it); no more CTAs than about one per 8 triangles.
    long long blocks = static_cast<long long>(sms) * per_sm;
    const long long want = (static_cast<long long>(a.triangles) + 7) / 8;
    if (blocks > want) blocks = want;
    if (blocks < 1) blocks = 1;
    void *args[] = {const_cast<MeshBuildArgs *>(&a), const_cast<MeshBuildScratch *>(&t), &slot_mesh, &slots, &mesh,
        &slot_root, &slot_bounds, &slot_hull};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(build_mesh_kernel), dim3(static_cast<unsigned>(blocks)),
        dim3(256), args, 0, stream);
}

}  // namespace ngb
