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

static void check_lights(const ngb_light *lights, int count) {
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
// The binned surface-area-heuristic build of src/bvh.cpp:46-174 (16 bins, leaf at most 4 triangles, depth
// at most 60), with the same tie rules, partition and node order, so every mesh gets the reference's tree
// node for node and its triangles in the reference's leaf order.

namespace {

struct Box {
    float lo[3], hi[3];
};

Box empty_box() {
    const float inf = std::numeric_limits<float>::infinity();
    return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}

void grow(Box &b, const Box &o) {
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = std::min(b.lo[k], o.lo[k]);
        b.hi[k] = std::max(b.hi[k], o.hi[k]);
    }
}

float area(const Box &b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct Node {
    float lo[3];
    int32_t a;
    float hi[3];
    int32_t count;
};

constexpr int BINS = 16;
constexpr int MAX_DEPTH = 60;

// Returns the nodes (root first) and fills order with the primitives in leaf order.
std::vector<Node> sah_build(const std::vector<Box> &bounds, std::vector<uint32_t> &order) {
    const uint32_t n = static_cast<uint32_t>(bounds.size());
    std::vector<Node> nodes;
    order.resize(n);
    if (n == 0) return nodes;
    std::iota(order.begin(), order.end(), 0u);
    std::vector<std::array<float, 3>> centre(n);
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) centre[i][k] = 0.5f * (bounds[i].lo[k] + bounds[i].hi[k]);
    nodes.reserve(2 * static_cast<size_t>(n));
    nodes.emplace_back();
    struct Work {
        int node;
        uint32_t begin, end;
        int depth;
    };
    std::vector<Work> stack{{0, 0, n, 0}};
    auto bin_of = [](float c, float lo, float scale) { return std::min(BINS - 1, static_cast<int>((c - lo) * scale)); };
    while (!stack.empty()) {
        const Work wk = stack.back();
        stack.pop_back();
        const uint32_t count = wk.end - wk.begin;
        uint32_t *prims = order.data() + wk.begin;
        Box box = empty_box(), cbox = empty_box();
        for (uint32_t i = 0; i < count; ++i) {
            grow(box, bounds[prims[i]]);
            for (int k = 0; k < 3; ++k) {
                cbox.lo[k] = std::min(cbox.lo[k], centre[prims[i]][k]);
                cbox.hi[k] = std::max(cbox.hi[k], centre[prims[i]][k]);
            }
        }
        Node node{};
        for (int k = 0; k < 3; ++k) {
            node.lo[k] = box.lo[k];
            node.hi[k] = box.hi[k];
        }
        int best_axis = -1, best_bin = 0;
        float best_cost = std::numeric_limits<float>::infinity();
        if (count > 1) {
            for (int axis = 0; axis < 3; ++axis) {
                const float extent = cbox.hi[axis] - cbox.lo[axis];
                if (!(extent > 0.0f)) continue;
                const float scale = static_cast<float>(BINS) / extent;
                int bin_count[BINS] = {};
                Box bin_box[BINS];
                for (Box &b : bin_box) b = empty_box();
                for (uint32_t i = 0; i < count; ++i) {
                    const int b = bin_of(centre[prims[i]][axis], cbox.lo[axis], scale);
                    ++bin_count[b];
                    grow(bin_box[b], bounds[prims[i]]);
                }
                float right_area[BINS - 1];
                int right_count[BINS - 1];
                Box acc = empty_box();
                int running = 0;
                for (int i = BINS - 1; i >= 1; --i) {
                    grow(acc, bin_box[i]);
                    running += bin_count[i];
                    right_area[i - 1] = area(acc);
                    right_count[i - 1] = running;
                }
                acc = empty_box();
                running = 0;
                for (int i = 0; i < BINS - 1; ++i) {
                    grow(acc, bin_box[i]);
                    running += bin_count[i];
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
        const bool small = count <= 4u;
        if (count == 1 || wk.depth >= MAX_DEPTH || (small && (best_axis < 0 || leaf_cost <= split_cost))) {
            node.a = static_cast<int32_t>(wk.begin);
            node.count = static_cast<int32_t>(count);
            nodes[wk.node] = node;
            continue;
        }
        uint32_t mid;
        if (best_axis >= 0) {
            const float lo = cbox.lo[best_axis];
            const float scale = static_cast<float>(BINS) / (cbox.hi[best_axis] - lo);
            const uint32_t *p = std::partition(prims, prims + count,
                [&](uint32_t prim) { return bin_of(centre[prim][best_axis], lo, scale) <= best_bin; });
            mid = wk.begin + static_cast<uint32_t>(p - prims);
            if (mid == wk.begin || mid == wk.end) mid = wk.begin + count / 2;
        } else {
            mid = wk.begin + count / 2;
        }
        const int left = static_cast<int>(nodes.size());
        nodes.resize(nodes.size() + 2);
        node.a = left;
        node.count = 0;
        nodes[wk.node] = node;
        stack.push_back({left + 1, mid, wk.end, wk.depth + 1});
        stack.push_back({left, wk.begin, mid, wk.depth + 1});
    }
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
        std::vector<Box> tri_bounds(tri_count);
        for (size_t t = 0; t < tri_count; ++t) {
            Box b = empty_box();
            for (int k = 0; k < 3; ++k) {
                const float *v = mesh.vertices + 3 * static_cast<size_t>(mesh.indices[3 * t + k]);
                for (int a = 0; a < 3; ++a) {
                    b.lo[a] = std::fmin(b.lo[a], v[a]);
                    b.hi[a] = std::fmax(b.hi[a], v[a]);
                }
            }
            tri_bounds[t] = b;
        }
        std::vector<uint32_t> order;
        const std::vector<Node> tree = sah_build(tri_bounds, order);
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
