// Host-side pieces of the renderer: input validation (with the reference's messages) and the meshes'
// bottom-level trees. No CUDA here.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <array>
#include <string>
#include <vector>

#include "../../include/ngb.h"

namespace ngb {

// A rejected argument: NGB_INVALID_ARGUMENT, std::invalid_argument in the reference.
struct InvalidArgument : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
// A failed CUDA call: NGB_CUDA_ERROR, neraulgraphics::CudaError in the reference.
struct CudaFailure : std::runtime_error {
    int code;
    CudaFailure(int c, const std::string &what) : std::runtime_error(what), code(c) {}
};
// A bounded device wait that ran out: NGB_TIMEOUT.
struct Timeout : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void require(bool ok, const std::string &message);
bool finite(float v);
bool all_finite(const float *v, size_t count);
std::string fstr(float v);  // std::to_string(float): "%f"

void check_frame_size(int width, int height);                          // src/validate.cpp:34-40
void check_scene(const ngb_scene &s);                                   // src/validate.cpp:61-78, 42-59
void check_lights(const ngb_light *lights, int count);                  // src/validate.cpp:41-59
void check_meshes(const ngb_scene &s);                                  // src/mesh_build.cpp:31-89
void check_material(const ngb_material &m, const std::string &name);   // src/validate.cpp:22-31
bool invert_affine(const float *m, float *out);                         // src/mesh_build.cpp:159-183
bool transform_ok(const float *m);                                      // src/mesh_build.cpp:18-23
void check_transform(const float *m, const std::string &name);          // src/mesh_build.cpp:25-29
bool quaternion_is_usable(const float *q);                              // src/batch.cpp:29-32
void check_environment(const ngb_environment &e);                       // src/environment.cpp:9-27

// Every mesh's tree, concatenated (src/mesh_build.h:16-29): nodes as bvh::Node (lo.xyz, a, hi.xyz, count),
// triangles in leaf order as v0, e1, e2 padded to float4, per-triangle vertex normals when any mesh has
// them, each packed triangle's index in its own mesh, and per mesh its root and its box in its own space.
struct BuiltMeshes {
    std::vector<float> nodes;        // 8 words per node (a and count stored as int bits)
    std::vector<float> triangles;    // 12 per triangle
    std::vector<float> attributes;   // 16 per triangle, or empty
    std::vector<int32_t> triangle_index;
    std::vector<int32_t> roots;
    std::vector<float> bounds;       // 6 per mesh
    // The same trees as child-pair records, one per node (used for internal nodes only): both children's
    // boxes and references in 64 bytes, (c0.lo.xyz, c0.hi.x) (c0.hi.yz, c1.lo.xy) (c1.lo.z, c1.hi.xyz)
    // (c0.ref, c0.count, c1.ref, c1.count). A reference is (node, 0) for an internal child and (first
    // triangle, count) for a leaf. Per mesh, its root's reference.
    std::vector<float> pairs;        // 16 per node
    std::vector<int32_t> root_refs;  // 2 per mesh
    std::vector<int32_t> node_counts;  // per mesh: its tree's nodes
};

// node_capacity: with it, mesh m's nodes start at the sum of the capacities 2 T_k - 1 of the meshes before it
// (T_k triangles) and its unused capacity is zero nodes, so a tree rebuilt on the device for new vertex
// positions (which may have another node count, never above 2 T - 1) fits where the first one was.
BuiltMeshes build_meshes(const ngb_scene &s, bool node_capacity = false);

// A mesh's hull facts for the shadow rays: the vertices' mean (x, y, z) and, in w, their largest distance from
// it when the mesh is convex (every vertex on the mean's side of every triangle's plane, within 1e-6 of that
// distance, and the mean at least 1e-3 of it inside), else -1. Meshes above 2^25 triangle-vertex pairs are
// not checked (-1).
std::array<float, 4> mesh_hull(const ngb_mesh &mesh);

// A sphere holding every vertex of the mesh (so every triangle): the vertices' mean (x, y, z) rounded to float, and
// in w their largest distance from that point, rounded up; -1 for a mesh without vertices.
std::array<float, 4> mesh_sphere(const ngb_mesh &mesh);

// The sRGB byte of a linear value, (uint8)(saturate(srgb(saturate(v))) * 255 + 0.5) with srgb's 1/2.4 power
// taken by the host's powf (src/geom_dev.h:169-182, render_core.h:280-282), as 255 thresholds: t[k] (k = 1..255)
// is the smallest float whose byte is k or more, t[0] = 0. The byte of v is the number of k >= 1 with
// t[k] <= v. Found by bisection over the floats of [0, 1] (the mapping is monotonic there).
void srgb_thresholds(float t[256]);
uint8_t srgb_byte(float v);  // the mapping itself, on the host

}  // namespace ngb
