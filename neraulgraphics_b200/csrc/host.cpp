// Validation and the meshes' bottom-level trees, on the host. Built without -ffast-math so the NaN checks
// stand (src/validate.h:1-6).
#include "host.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>

namespace ngb {

void require(bool ok, const std::string &message) {
    if (!ok) throw InvalidArgument(message);
}

bool finite(float v) { return std::isfinite(v); }

bool all_finite(const float *v, size_t count) {
    for (size_t i = 0; i < count; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

std::string fstr(float v) { return std::to_string(v); }

static bool finite3(const ngb_vec3 &v) { return finite(v.x) && finite(v.y) && finite(v.z); }

void check_material(const ngb_material &m, const std::string &name) {
    const bool ok = finite3(m.diffuse_color) && finite(m.diffuse_albedo) && finite(m.specular_albedo) &&
        finite(m.reflectivity) && finite(m.specular_exponent) && finite(m.roughness) && finite(m.metallic) &&
        finite3(m.emission) && finite(m.transmission) && finite(m.ior);
    require(ok, name + " has a NaN or infinite value");
    require(m.roughness <= 1.0f, name + " roughness must be at most 1, got " + fstr(m.roughness));
    require(m.metallic <= 1.0f, name + " metallic must be at most 1, got " + fstr(m.metallic));
    require(m.emission.x >= 0.0f && m.emission.y >= 0.0f && m.emission.z >= 0.0f, name + " emission must not be negative");
    require(m.transmission >= 0.0f && m.transmission <= 1.0f, name + " transmission must be 0 to 1, got " + fstr(m.transmission));
    require(m.ior >= 1.0f && m.ior <= 4.0f, name + " ior must be 1 to 4, got " + fstr(m.ior));
}

void check_frame_size(int width, int height) {
    require(width > 0 && height > 0, "frame size must be positive, got " + std::to_string(width) + "x" +
        std::to_string(height));
    require(static_cast<long long>(width) * height <= INT32_MAX,
        "frame of " + std::to_string(width) + "x" + std::to_string(height) + " pixels is too large");
}

void check_lights(const ngb_light *lights, int count) {
    require(count <= NGB_MAX_LIGHTS, "scene has " + std::to_string(count) + " lights, at most " +
        std::to_string(NGB_MAX_LIGHTS) + " fit");
    for (int i = 0; i < count; ++i) {
        const ngb_light &l = lights[i];
        const std::string name = "light " + std::to_string(i);
        require(finite3(l.position) && finite(l.intensity) && finite(l.radius), name + " has a NaN or infinite value");
        require(l.radius >= 0.0f, name + " radius must be 0 or more, got " + fstr(l.radius));
        require(finite(l.falloff) && l.falloff >= 0.0f, name + " falloff must be 0 or more, got " + fstr(l.falloff));
        require(finite3(l.direction) && finite(l.spot_angle) && finite(l.spot_softness), name + " has a NaN or infinite value");
        require(l.spot_angle >= 0.0f && l.spot_angle < 3.14159f,
            name + " spot_angle must be 0 (no cone) to below pi radians, got " + fstr(l.spot_angle));
        require(finite3(l.color) && l.color.x >= 0.0f && l.color.y >= 0.0f && l.color.z >= 0.0f,
            name + " color must be finite and not negative");
        require(l.spot_softness >= 0.0f && l.spot_softness <= 1.0f, name + " spot_softness must be 0 to 1, got " + fstr(l.spot_softness));
        require(l.spot_angle == 0.0f || l.direction.x != 0.0f || l.direction.y != 0.0f || l.direction.z != 0.0f,
            name + " is a spotlight (spot_angle > 0) but its direction is zero");
    }
}

void check_scene(const ngb_scene &s) {
    require(s.sphere_count >= 0 && s.light_count >= 0 && s.mesh_count >= 0 && s.instance_count >= 0,
        "counts must not be negative");
    require(s.sphere_count <= NGB_MAX_SPHERES, "scene has " + std::to_string(s.sphere_count) + " spheres, at most " +
        std::to_string(NGB_MAX_SPHERES) + " fit");
    require(s.light_count == 0 || s.lights != nullptr, "lights must not be null");
    require(s.sphere_count == 0 || s.spheres != nullptr, "spheres must not be null");
    check_lights(s.lights, s.light_count);
    for (int i = 0; i < s.sphere_count; ++i) {
        const ngb_sphere &sp = s.spheres[i];
        const std::string name = "sphere " + std::to_string(i);
        require(finite3(sp.center) && finite(sp.radius), name + " has a NaN or infinite value");
        check_material(sp.material, name);
        require(sp.radius > 0.0f, name + " radius must be positive, got " + fstr(sp.radius));
    }
    const ngb_plane &f = s.floor;
    require(finite(f.y) && finite(f.half_extent_x) && finite(f.z_min) && finite(f.z_max) && finite(f.checker_scale),
        "floor has a NaN or infinite value");
    check_material(f.material, "floor");
}

bool invert_affine(const float *m, float *out) {
    const float c00 = m[5] * m[10] - m[6] * m[9];
    const float c01 = m[6] * m[8] - m[4] * m[10];
    const float c02 = m[4] * m[9] - m[5] * m[8];
    const float det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    float mag = 0.0f;
    for (const int i : {0, 1, 2, 4, 5, 6, 8, 9, 10}) mag = std::fmax(mag, std::fabs(m[i]));
    if (!std::isfinite(det) || std::fabs(det) <= 1e-12f * mag * mag * mag) return false;
    const float inv = 1.0f / det;
    const float r[9] = {c00 * inv, (m[2] * m[9] - m[1] * m[10]) * inv, (m[1] * m[6] - m[2] * m[5]) * inv, c01 * inv,
        (m[0] * m[10] - m[2] * m[8]) * inv, (m[2] * m[4] - m[0] * m[6]) * inv, c02 * inv,
        (m[1] * m[8] - m[0] * m[9]) * inv, (m[0] * m[5] - m[1] * m[4]) * inv};
    for (int row = 0; row < 3; ++row) {
        for (int col = 0; col < 3; ++col) out[4 * row + col] = r[3 * row + col];
        out[4 * row + 3] = -(r[3 * row] * m[3] + r[3 * row + 1] * m[7] + r[3 * row + 2] * m[11]);
    }
    return true;
}

bool transform_ok(const float *m) {
    for (int k = 0; k < 12; ++k)
        if (!finite(m[k])) return false;
    float inv[12];
    return invert_affine(m, inv);
}

void check_transform(const float *m, const std::string &name) {
    for (int k = 0; k < 12; ++k) require(finite(m[k]), name + " has a NaN or infinite value");
    float inv[12];
    require(invert_affine(m, inv), name + " is singular (it flattens space, so it cannot be inverted)");
}

bool quaternion_is_usable(const float *q) {
    return finite(q[0]) && finite(q[1]) && finite(q[2]) && finite(q[3]) &&
        q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3] > 0.0f;
}

void check_meshes(const ngb_scene &s) {
    require(s.mesh_count == 0 || s.meshes != nullptr, "meshes must not be null");
    require(s.instance_count == 0 || s.instances != nullptr, "instances must not be null");
    constexpr size_t MAX_TRIANGLES = 100000000;
    for (int m = 0; m < s.mesh_count; ++m) {
        const ngb_mesh &mesh = s.meshes[m];
        const std::string name = "mesh " + std::to_string(m);
        require(mesh.vertex_count >= 0 && mesh.index_count >= 0, name + " has a negative count");
        require(mesh.index_count > 0, name + " has no triangles");
        require(mesh.index_count % 3 == 0, name + " has " + std::to_string(mesh.index_count) +
            " indices, which is not a multiple of 3");
        require(static_cast<size_t>(mesh.index_count) / 3 <= MAX_TRIANGLES, name + " has too many triangles");
        for (int i = 0; i < mesh.vertex_count; ++i)
            require(finite(mesh.vertices[3 * i]) && finite(mesh.vertices[3 * i + 1]) && finite(mesh.vertices[3 * i + 2]),
                name + " vertex " + std::to_string(i) + " has a NaN or infinite value");
        if (mesh.normals)
            for (int i = 0; i < mesh.vertex_count; ++i)
                require(finite(mesh.normals[3 * i]) && finite(mesh.normals[3 * i + 1]) && finite(mesh.normals[3 * i + 2]),
                    name + " normal " + std::to_string(i) + " has a NaN or infinite value");
        for (int i = 0; i < mesh.index_count; ++i)
            require(mesh.indices[i] < static_cast<uint32_t>(mesh.vertex_count), name + " index " + std::to_string(i) +
                " is " + std::to_string(mesh.indices[i]) + ", but there are only " + std::to_string(mesh.vertex_count) +
                " vertices");
    }
    for (int i = 0; i < s.instance_count; ++i) {
        const ngb_instance &inst = s.instances[i];
        const std::string name = "instance " + std::to_string(i);
        require(inst.mesh >= 0 && inst.mesh < s.mesh_count, name + " uses mesh " + std::to_string(inst.mesh) +
            ", but there are " + std::to_string(s.mesh_count) + " meshes");
        check_transform(inst.transform, name + " transform");
        check_material(inst.material, name + " material");
    }
}

void check_environment(const ngb_environment &e) {
    require(finite3(e.up) && e.up.x * e.up.x + e.up.y * e.up.y + e.up.z * e.up.z > 1e-12f,
        "environment up must be a nonzero vector with no NaN or infinite value");
    for (const ngb_vec3 &c : {e.color_up, e.color_down})
        require(finite3(c) && c.x >= 0.0f && c.y >= 0.0f && c.z >= 0.0f, "environment colours must be finite and not negative");
    require(finite(e.intensity) && e.intensity >= 0.0f, "environment intensity must be 0 or more, got " + fstr(e.intensity));
}

// ----------------------------------------------------------------------------- bottom-level trees --
//
// Each mesh's tree is the binned surface-area-heuristic tree of src/bvh.cpp:46-174 (16 bins, leaves of at
// most 4 triangles, depth at most 60), node for node, with its triangles in the same leaf order. It is built
// the way the device rebuild in blas_build.cu builds it, so the two builders are one algorithm:
//   - level by level: every node of a depth is split before any node of the next depth; a node's children are
//     appended to the next depth's list (a split's outcome depends only on its own triangle range, so the
//     order in which nodes are split does not change the tree);
//   - a split moves its range's triangles with the swaps std::partition (libstdc++'s bidirectional form)
//     makes: the k-th triangle from the left that fails the test trades places with the k-th from the right
//     that passes it, for every k before the two runs meet;
//   - the numbering comes last, in closed form: the reference numbers a node's children 2k + 1 and 2k + 2 when
//     it splits the k-th internal node in depth-first, left-first order, and an internal node's k is the count
//     of internal nodes starting (in leaf order) before it plus its depth below the topmost internal node that
//     starts where it starts.

namespace {

struct Box {
    float lo[3], hi[3];
};

constexpr float INF = std::numeric_limits<float>::infinity();
constexpr int BINS = 16;
constexpr uint32_t MAX_LEAF = 4;
constexpr int MAX_DEPTH = 60;

// Box arithmetic with the reference's tie rule: of two equal values (only -0 and +0 differ) the earlier in
// range order is kept, as std::min / std::max keep their first argument.
void take(Box &b, const float *lo, const float *hi) {
    for (int k = 0; k < 3; ++k) {
        if (lo[k] < b.lo[k]) b.lo[k] = lo[k];
        if (b.hi[k] < hi[k]) b.hi[k] = hi[k];
    }
}

float surface(const Box &b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

int bin_index(float c, float lo, float scale) {
    const int b = static_cast<int>((c - lo) * scale);
    return b < BINS - 1 ? b : BINS - 1;
}

// A node while the tree is built: its triangle range in `order`, its depth, its box and its first child in
// level order (-1 for a leaf).
struct Draft {
    uint32_t begin, end;
    int depth;
    int first_child;
    Box box;
};

// The triangles of one mesh: their boxes (6 floats) and centroids (3 floats), and their order.
struct Items {
    std::vector<float> box, centre;
    std::vector<uint32_t> order;
};

// The cheapest split plane of a range, over the axes in order (src/bvh.cpp:94-125): axis -1 when no axis
// has spread centroids or no plane leaves triangles on both sides.
struct Plane {
    int axis = -1, bin = 0;
    float cost = INF;
};

Plane cheapest_plane(const Items &it, uint32_t begin, uint32_t end, const Box &cbox) {
    Plane best;
    for (int axis = 0; axis < 3; ++axis) {
        const float extent = cbox.hi[axis] - cbox.lo[axis];
        if (!(extent > 0.0f)) continue;
        const float scale = static_cast<float>(BINS) / extent;
        Box bins[BINS];
        int count[BINS] = {};
        for (Box &b : bins) b = Box{{INF, INF, INF}, {-INF, -INF, -INF}};
        for (uint32_t i = begin; i < end; ++i) {
            const float *tb = &it.box[6 * static_cast<size_t>(it.order[i])];
            const int b = bin_index(it.centre[3 * static_cast<size_t>(it.order[i]) + axis], cbox.lo[axis], scale);
            ++count[b];
            take(bins[b], tb, tb + 3);
        }
        // Suffix areas and counts: plane p separates bins [0, p] from [p + 1, BINS).
        float suffix_area[BINS];
        int suffix_count[BINS];
        Box acc{{INF, INF, INF}, {-INF, -INF, -INF}};
        int n = 0;
        for (int b = BINS - 1; b >= 1; --b) {
            take(acc, bins[b].lo, bins[b].hi);
            n += count[b];
            suffix_area[b] = surface(acc);
            suffix_count[b] = n;
        }
        acc = Box{{INF, INF, INF}, {-INF, -INF, -INF}};
        n = 0;
        for (int p = 0; p + 1 < BINS; ++p) {
            take(acc, bins[p].lo, bins[p].hi);
            n += count[p];
            if (n == 0 || suffix_count[p + 1] == 0) continue;
            const float cost = static_cast<float>(n) * surface(acc) +
                static_cast<float>(suffix_count[p + 1]) * suffix_area[p + 1];
            if (cost < best.cost) best = Plane{axis, p, cost};
        }
    }
    return best;
}

// Splits drafts[x]: fills its box and, unless it stays a leaf, partitions its range and appends its two
// children to `drafts` (src/bvh.cpp:62-170).
void split(Items &it, std::vector<Draft> &drafts, size_t x) {
    const uint32_t begin = drafts[x].begin, end = drafts[x].end, count = end - begin;
    const int depth = drafts[x].depth;
    Box box{{INF, INF, INF}, {-INF, -INF, -INF}}, cbox = box;
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t p = it.order[i];
        take(box, &it.box[6 * static_cast<size_t>(p)], &it.box[6 * static_cast<size_t>(p) + 3]);
        const float *c = &it.centre[3 * static_cast<size_t>(p)];
        take(cbox, c, c);
    }
    drafts[x].box = box;
    drafts[x].first_child = -1;
    const Plane plane = count > 1 ? cheapest_plane(it, begin, end, cbox) : Plane{};
    const float here = surface(box);
    const bool leaf = count == 1 || depth >= MAX_DEPTH ||
        (count <= MAX_LEAF && (plane.axis < 0 || static_cast<float>(count) * here <= 1.0f * here + plane.cost));
    if (leaf) return;
    uint32_t mid = begin + count / 2;
    if (plane.axis >= 0) {
        const float lo = cbox.lo[plane.axis];
        const float scale = static_cast<float>(BINS) / (cbox.hi[plane.axis] - lo);
        auto passes = [&](uint32_t i) {
            return bin_index(it.centre[3 * static_cast<size_t>(it.order[i]) + plane.axis], lo, scale) <= plane.bin;
        };
        uint32_t meet = begin;
        for (uint32_t i = begin; i < end; ++i) meet += passes(i) ? 1u : 0u;
        // The k-th failing position left of meet and the k-th passing position right of it, from the right.
        std::vector<uint32_t> fail_left, pass_right;
        for (uint32_t i = begin; i < meet; ++i)
            if (!passes(i)) fail_left.push_back(i);
        for (uint32_t j = end; j-- > meet;)
            if (passes(j)) pass_right.push_back(j);
        for (size_t k = 0; k < fail_left.size(); ++k) std::swap(it.order[fail_left[k]], it.order[pass_right[k]]);
        mid = meet;
        if (mid == begin || mid == end) mid = begin + count / 2;
    }
    drafts[x].first_child = static_cast<int>(drafts.size());
    drafts.push_back(Draft{begin, mid, depth + 1, -1, {}});
    drafts.push_back(Draft{mid, end, depth + 1, -1, {}});
}

struct Node {
    float lo[3];
    int32_t a;
    float hi[3];
    int32_t count;
};

// The tree over the triangle boxes `tri_box` (6 floats each): nodes in the reference's numbering (root first)
// with mesh-local references, and `order` the triangles in leaf order.
std::vector<Node> build_tree(std::vector<float> tri_box, std::vector<uint32_t> &order) {
    Items it;
    const uint32_t n = static_cast<uint32_t>(tri_box.size() / 6);
    it.box = std::move(tri_box);
    it.centre.resize(3 * static_cast<size_t>(n));
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) it.centre[3 * i + k] = 0.5f * (it.box[6 * i + k] + it.box[6 * i + 3 + k]);
    it.order.resize(n);
    std::iota(it.order.begin(), it.order.end(), 0u);
    std::vector<Node> nodes;
    if (n == 0) {
        order.clear();
        return nodes;
    }
    std::vector<Draft> drafts{Draft{0, n, 0, -1, {}}};
    drafts.reserve(2 * static_cast<size_t>(n));
    for (size_t first = 0, last = 1; first < last; first = last, last = drafts.size())
        for (size_t x = first; x < last; ++x) split(it, drafts, x);

    // Closed-form numbering of the depth-first order.
    std::vector<int> starts(n + 1, 0), top(n, INT_MAX);
    for (const Draft &d : drafts)
        if (d.first_child >= 0) {
            ++starts[d.begin + 1];
            top[d.begin] = std::min(top[d.begin], d.depth);
        }
    for (uint32_t i = 0; i < n; ++i) starts[i + 1] += starts[i];  // internal nodes starting before i
    std::vector<int> index(drafts.size(), 0);
    for (const Draft &d : drafts) {
        if (d.first_child < 0) continue;
        const int k = starts[d.begin] + d.depth - top[d.begin];
        index[d.first_child] = 2 * k + 1;
        index[d.first_child + 1] = 2 * k + 2;
    }
    nodes.resize(drafts.size());
    for (size_t x = 0; x < drafts.size(); ++x) {
        const Draft &d = drafts[x];
        Node &nd = nodes[index[x]];
        for (int k = 0; k < 3; ++k) {
            nd.lo[k] = d.box.lo[k];
            nd.hi[k] = d.box.hi[k];
        }
        const bool leaf = d.first_child < 0;
        nd.a = leaf ? static_cast<int32_t>(d.begin) : index[d.first_child];
        nd.count = leaf ? static_cast<int32_t>(d.end - d.begin) : 0;
    }
    order = std::move(it.order);
    return nodes;
}

}  // namespace

BuiltMeshes build_meshes(const ngb_scene &s, bool node_capacity) {
    BuiltMeshes out;
    bool any_normals = false;
    for (int m = 0; m < s.mesh_count; ++m) any_normals = any_normals || s.meshes[m].normals != nullptr;
    for (int m = 0; m < s.mesh_count; ++m) {
        const ngb_mesh &mesh = s.meshes[m];
        const size_t tri_count = static_cast<size_t>(mesh.index_count) / 3;
        // Triangle boxes over the vertices in order; of two equal values (-0 and +0) the later is kept, as the
        // reference's std::fmin / std::fmax give them (src/mesh_build.cpp:98-110).
        std::vector<float> tri_box(6 * tri_count);
        for (size_t t = 0; t < tri_count; ++t) {
            float *b = &tri_box[6 * t];
            for (int a = 0; a < 3; ++a) {
                b[a] = INF;
                b[3 + a] = -INF;
            }
            for (int k = 0; k < 3; ++k) {
                const float *v = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t + k]);
                for (int a = 0; a < 3; ++a) {
                    b[a] = b[a] < v[a] ? b[a] : v[a];
                    b[3 + a] = b[3 + a] > v[a] ? b[3 + a] : v[a];
                }
            }
        }
        std::vector<uint32_t> order;
        const std::vector<Node> tree = build_tree(std::move(tri_box), order);
        const int node_base = static_cast<int>(out.nodes.size() / 8);
        const int tri_base = static_cast<int>(out.triangles.size() / 12);
        out.roots.push_back(node_base);
        out.bounds.insert(out.bounds.end(), {tree[0].lo[0], tree[0].lo[1], tree[0].lo[2], tree[0].hi[0], tree[0].hi[1],
            tree[0].hi[2]});
        for (Node nd : tree) {
            nd.a += nd.count > 0 ? tri_base : node_base;
            float words[8];
            std::memcpy(words, &nd, sizeof(words));
            out.nodes.insert(out.nodes.end(), words, words + 8);
        }
        auto ref_of = [&](const Node &nd, int index) {
            return nd.count > 0 ? std::array<int32_t, 2>{nd.a + tri_base, nd.count} : std::array<int32_t, 2>{index + node_base, 0};
        };
        for (size_t i = 0; i < tree.size(); ++i) {
            float rec[16] = {};
            const Node &nd = tree[i];
            if (nd.count == 0) {
                const Node &l = tree[nd.a], &r = tree[nd.a + 1];
                const std::array<int32_t, 2> lr = ref_of(l, nd.a), rr = ref_of(r, nd.a + 1);
                const float v[12] = {l.lo[0], l.lo[1], l.lo[2], l.hi[0], l.hi[1], l.hi[2], r.lo[0], r.lo[1], r.lo[2],
                    r.hi[0], r.hi[1], r.hi[2]};
                std::memcpy(rec, v, sizeof(v));
                const int32_t refs[4] = {lr[0], lr[1], rr[0], rr[1]};
                std::memcpy(rec + 12, refs, sizeof(refs));
            }
            out.pairs.insert(out.pairs.end(), rec, rec + 16);
        }
        const std::array<int32_t, 2> root = ref_of(tree[0], 0);
        out.root_refs.insert(out.root_refs.end(), root.begin(), root.end());
        out.node_counts.push_back(static_cast<int32_t>(tree.size()));
        if (node_capacity) {
            const size_t cap = 2 * tri_count - 1;
            out.nodes.resize(out.nodes.size() + 8 * (cap - tree.size()), 0.0f);
            out.pairs.resize(out.pairs.size() + 16 * (cap - tree.size()), 0.0f);
        }
        for (const uint32_t t : order) {
            const float *a = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t]);
            const float *b = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t + 1]);
            const float *c = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t + 2]);
            out.triangles.insert(out.triangles.end(), {a[0], a[1], a[2], 0.0f, b[0] - a[0], b[1] - a[1], b[2] - a[2], 0.0f,
                c[0] - a[0], c[1] - a[1], c[2] - a[2], 0.0f});
            out.triangle_index.push_back(static_cast<int32_t>(t));
            if (any_normals) {
                float rec[16] = {};
                if (mesh.normals)
                    for (int k = 0; k < 3; ++k) {
                        const uint32_t vi = mesh.indices[3 * t + k];
                        rec[4 * k] = mesh.normals[3 * vi];
                        rec[4 * k + 1] = mesh.normals[3 * vi + 1];
                        rec[4 * k + 2] = mesh.normals[3 * vi + 2];
                    }
                const int32_t flags = mesh.normals ? 1 : 0;  // ATTR_NORMALS (src/mesh_build.h:28)
                std::memcpy(&rec[15], &flags, sizeof(flags));
                out.attributes.insert(out.attributes.end(), rec, rec + 16);
            }
        }
    }
    return out;
}

std::array<float, 4> mesh_hull(const ngb_mesh &mesh) {
    const int V = mesh.vertex_count, T = mesh.index_count / 3;
    double c[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < V; ++i)
        for (int k = 0; k < 3; ++k) c[k] += mesh.vertices[3 * i + k];
    for (int k = 0; k < 3; ++k) c[k] /= std::max(V, 1);
    double radius = 0.0;
    for (int i = 0; i < V; ++i) {
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k) d2 += (mesh.vertices[3 * i + k] - c[k]) * (mesh.vertices[3 * i + k] - c[k]);
        radius = std::max(radius, std::sqrt(d2));
    }
    std::array<float, 4> out = {static_cast<float>(c[0]), static_cast<float>(c[1]), static_cast<float>(c[2]), -1.0f};
    if (V == 0 || T == 0 || radius <= 0.0 || static_cast<double>(T) * V > 33554432.0) return out;
    for (int t = 0; t < T; ++t) {
        const float *a = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t]);
        const float *b = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t + 1]);
        const float *d = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t + 2]);
        const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
        double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (!(len > 0.0)) return out;  // a degenerate triangle: no plane to test against
        for (double &x : n) x /= len;
        const double side = (c[0] - a[0]) * n[0] + (c[1] - a[1]) * n[1] + (c[2] - a[2]) * n[2];
        if (std::fabs(side) < 1e-3 * radius) return out;
        const double s = side > 0.0 ? 1.0 : -1.0;
        for (int i = 0; i < V; ++i) {
            const float *v = mesh.vertices + 3 * static_cast<size_t>(i);
            const double h = ((v[0] - a[0]) * n[0] + (v[1] - a[1]) * n[1] + (v[2] - a[2]) * n[2]) * s;
            if (h < -1e-6 * radius) return out;
        }
    }
    out[3] = static_cast<float>(radius);
    return out;
}

std::array<float, 4> mesh_sphere(const ngb_mesh &mesh) {
    const int V = mesh.vertex_count;
    if (V <= 0) return {0.0f, 0.0f, 0.0f, -1.0f};
    double c[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < V; ++i)
        for (int k = 0; k < 3; ++k) c[k] += mesh.vertices[3 * i + k];
    for (int k = 0; k < 3; ++k) c[k] /= V;
    const float cf[3] = {static_cast<float>(c[0]), static_cast<float>(c[1]), static_cast<float>(c[2])};
    double radius = 0.0;  // from the float centre, as the kernels hold it
    for (int i = 0; i < V; ++i) {
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k) d2 += (mesh.vertices[3 * i + k] - static_cast<double>(cf[k])) *
            (mesh.vertices[3 * i + k] - static_cast<double>(cf[k]));
        radius = std::max(radius, std::sqrt(d2));
    }
    return {cf[0], cf[1], cf[2], static_cast<float>(radius * (1.0 + 1e-5) + 1e-30)};
}

uint8_t srgb_byte(float v) {
    const float x = std::fmin(std::fmax(v, 0.0f), 1.0f);
    const float c = x <= 0.0031308f ? 12.92f * x : 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f;
    return static_cast<uint8_t>(std::fmin(std::fmax(c, 0.0f), 1.0f) * 255.0f + 0.5f);
}

void srgb_thresholds(float t[256]) {
    t[0] = 0.0f;
    // Floats in [0, 1] are ordered like their bit patterns, so bisect on the bits.
    const uint32_t one = 0x3f800000u;
    for (int k = 1; k < 256; ++k) {
        uint32_t lo = 0, hi = one;  // byte(lo) < k <= byte(hi)
        while (hi - lo > 1) {
            const uint32_t mid = lo + (hi - lo) / 2;
            float m;
            std::memcpy(&m, &mid, 4);
            if (srgb_byte(m) >= k) hi = mid;
            else lo = mid;
        }
        std::memcpy(&t[k], &hi, 4);
    }
}

}  // namespace ngb
