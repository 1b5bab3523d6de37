// The adjoint of the depth and normal images with respect to the instance matrices and the camera matrices,
// visibility held fixed: every pixel keeps the (instance, triangle, barycentric) hit its centre ray recorded in
// the forward render, and the derivative is that of the same surface point as the matrices move.
//
// Forward quantities of a pixel (aov_pixel and mesh_surface, src/render_core.h:313-327, src/mesh_dev.h:238-262):
//   camera: right = c0 / |c0|, up = c1 / |c1|, forward f = -c2 / |c2|, eye o = c3 (c_k: the matrix's columns);
//           w = right sx + up sy + f, d = w / |w|
//   instance: world point X = A x + b; the hit's local point p = v0 + u e1 + v e2, world point P = o + t d
//   t = n . (A p + b - o) / (n . d) with n = A^-T (e1 x e2) the world geometric normal (any scale)
//   depth D = t (d . f); normal N = s m / |m| with m = A^-T n_s, n_s the local shading normal (the geometric
//   one, or the barycentric blend of the vertex normals), s = +-1 the forward's facing choice (held fixed).
// Their differentials, for a surface point that moves with the instance:
//   dt = [n . (dA p + db) - n . do - t n . dd] / (n . d)
//   d(A^-T) = -A^-T dA^T A^-T, dp = A^-1 (dP - dA p - db), (du, dv) = (a1 . dp, a2 . dp) with a1, a2 the dual
//   basis of (e1, e2) in the triangle's plane.
// The kernel applies their transposes to the upstream gradients of D and N, pixel by pixel, and sums them
// per instance and per camera: first in shared memory (one CTA is one 16 x 16 tile of one view, so all its
// pixels share a camera and a world), then into the caller's arrays with one atomic per entry and CTA.
#include "device.cuh"
#include "kernels.h"

namespace ngb {
namespace {

constexpr int ADJ_TILE = 16;
constexpr int ADJ_THREADS = ADJ_TILE * ADJ_TILE;

struct M3 {
    float a[3][3];
};

__device__ __forceinline__ float3 mul(const M3 &m, float3 v) {
    return mk3(m.a[0][0] * v.x + m.a[0][1] * v.y + m.a[0][2] * v.z, m.a[1][0] * v.x + m.a[1][1] * v.y + m.a[1][2] * v.z,
        m.a[2][0] * v.x + m.a[2][1] * v.y + m.a[2][2] * v.z);
}
__device__ __forceinline__ float3 mul_t(const M3 &m, float3 v) {  // m^T v
    return mk3(m.a[0][0] * v.x + m.a[1][0] * v.y + m.a[2][0] * v.z, m.a[0][1] * v.x + m.a[1][1] * v.y + m.a[2][1] * v.z,
        m.a[0][2] * v.x + m.a[1][2] * v.y + m.a[2][2] * v.z);
}
__device__ __forceinline__ void add_outer(M3 &g, float3 a, float3 b, float k) {
    const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) g.a[r][c] += k * av[r] * bv[c];
}
// The inverse of a 3 x 3 matrix by cofactors.
__device__ __forceinline__ M3 inverse(const M3 &m) {
    const float (*a)[3] = m.a;
    const float c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const float c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const float c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const float inv = 1.0f / (a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02);
    M3 r;
    r.a[0][0] = c00 * inv;
    r.a[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * inv;
    r.a[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * inv;
    r.a[1][0] = c01 * inv;
    r.a[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * inv;
    r.a[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * inv;
    r.a[2][0] = c02 * inv;
    r.a[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * inv;
    r.a[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * inv;
    return r;
}

// The gradient of x / |x| (x = v |v|): (g - n (n . g)) / |x|.
__device__ __forceinline__ float3 normalize_adjoint(float3 n, float len, float3 g) {
    return (g - n * dot(n, g)) * (1.0f / len);
}

// The camera's share: d = w / |w| with w = right sx + up sy + f, each basis vector its column normalised
// (f = -c2 / |c2|), the eye the last column; as the camera matrix's gradient (row-major 3 x 4).
__device__ __forceinline__ void camera_adjoint(float *gcam, float3 gdir, float3 gf, float3 go, float3 d, float lw,
    float3 right, float3 up, float3 f, float l0, float l1, float l2, float sx, float sy) {
    const float3 gw = normalize_adjoint(d, lw, gdir);
    const float3 gc0 = normalize_adjoint(right, l0, gw * sx);
    const float3 gc1 = normalize_adjoint(up, l1, gw * sy);
    const float3 gc2 = normalize_adjoint(f, l2, gw + gf) * -1.0f;
    const float g[12] = {gc0.x, gc1.x, gc2.x, go.x, gc0.y, gc1.y, gc2.y, go.y, gc0.z, gc1.z, gc2.z, go.z};
    for (int e = 0; e < 12; ++e) gcam[e] = g[e];
}

// The sum of v over the warp (every lane takes part), in every lane.
// Twelve sums over the warp at once (recursive halving): each exchange sends half of the values a lane still
// carries and keeps the other half, so 12 sums (padded to 16) take 8 + 4 + 2 + 1 + 1 shuffles instead of 12 x 5.
// Lane l ends with the total of entry l >> 1 (entries 12 to 15 are padding).
__device__ __forceinline__ float warp_sums12(const float *in, int lane) {
    float v[8];
    const bool b16 = lane & 16;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float lo = in[k], hi = k + 8 < 12 ? in[k + 8] : 0.0f;
        v[k] = (b16 ? hi : lo) + __shfl_xor_sync(0xffffffffu, b16 ? lo : hi, 16);
    }
    const bool b8 = lane & 8;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = (b8 ? v[k + 4] : v[k]) + __shfl_xor_sync(0xffffffffu, b8 ? v[k] : v[k + 4], 8);
    const bool b4 = lane & 4;
#pragma unroll
    for (int k = 0; k < 2; ++k) v[k] = (b4 ? v[k + 2] : v[k]) + __shfl_xor_sync(0xffffffffu, b4 ? v[k] : v[k + 2], 4);
    const bool b2 = lane & 2;
    v[0] = (b2 ? v[1] : v[0]) + __shfl_xor_sync(0xffffffffu, b2 ? v[0] : v[1], 2);
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

__global__ void __launch_bounds__(ADJ_THREADS, 4) depth_normal_adjoint_kernel(const __grid_constant__ SceneParams s,
    const AdjointArgs a, int tiles_x, int tiles_per_view, bool shared_sums) {
    extern __shared__ float sums[];  // per instance of the world 12, then the camera's 12
    const int view = blockIdx.x / tiles_per_view;
    const int q = blockIdx.x % tiles_per_view;
    const int x = (q % tiles_x) * ADJ_TILE + threadIdx.x % ADJ_TILE;
    const int y = a.row_first + (q / tiles_x) * ADJ_TILE + threadIdx.x / ADJ_TILE;
    const int world = view / a.cameras_per_world;
    const int P = s.per_world;
    float *cam_sum = sums + (shared_sums ? 12 * P : 0);
    for (int k = threadIdx.x; k < (shared_sums ? 12 * P : 0) + 12; k += ADJ_THREADS) sums[k] = 0.0f;
    __syncthreads();

    const long long pix = (static_cast<long long>(view) * a.rows + (y - a.row_first)) * a.width + x;
    const bool inside = x < a.width && y < a.row_first + a.rows;
    const int inst = inside ? a.hit_instance[pix] : -1;
    const float depth = inside ? a.depth[pix] : __int_as_float(0x7f800000);
    const bool hit = inside && isfinite(depth);
    const float gd = hit ? a.grad_depth[pix] : 0.0f;
    const float3 gn = hit && a.grad_normal
        ? mk3(a.grad_normal[3 * pix], a.grad_normal[3 * pix + 1], a.grad_normal[3 * pix + 2])
        : mk3(0.0f, 0.0f, 0.0f);
    float gcam[12], ginst[12];
    for (int e = 0; e < 12; ++e) gcam[e] = ginst[e] = 0.0f;
    int owner = -1;  // the instance ginst belongs to, -1 for none
    if (hit && (gd != 0.0f || gn.x != 0.0f || gn.y != 0.0f || gn.z != 0.0f)) {
        // The camera and the pixel's centre ray (camera_from_matrix, camera_ray).
        const float *cm = a.cameras + 12LL * view;
        const float3 c0 = mk3(cm[0], cm[4], cm[8]), c1 = mk3(cm[1], cm[5], cm[9]), c2 = mk3(cm[2], cm[6], cm[10]);
        const float3 o = mk3(cm[3], cm[7], cm[11]);
        const float l0 = sqrtf(dot(c0, c0)), l1 = sqrtf(dot(c1, c1)), l2 = sqrtf(dot(c2, c2));
        const float3 right = c0 * (1.0f / l0), up = c1 * (1.0f / l1), f = c2 * (-1.0f / l2);
        const float sx = (2.0f * (static_cast<float>(x) + 0.5f) / static_cast<float>(a.width) - 1.0f) * a.fov_scale * a.aspect;
        const float sy = -(2.0f * (static_cast<float>(y) + 0.5f) / static_cast<float>(a.height) - 1.0f) * a.fov_scale;
        const float3 w = right * sx + up * sy + f;
        const float lw = sqrtf(dot(w, w));
        const float3 d = w * (1.0f / lw);
        const float df = dot(d, f);
        const float t = depth / df;
        float3 go = mk3(0.0f, 0.0f, 0.0f), gdir = go, gf = go;
        if (inst < 0) {
            // Not a mesh: the floor (y = floor.y, normal constant) moves only with the camera; spheres carry no
            // gradient. t = (floor.y - o.y) / d.y, D = t (d . f).
            const float py = o.y + t * d.y;
            if (fabsf(d.y) > 1e-3f && fabsf(py - s.floor.y) <= 1e-4f * (1.0f + fabsf(s.floor.y) + fabsf(t))) {
                const float gt = gd * df;
                gdir = f * (gd * t);
                gf = d * (gd * t);
                go.y -= gt / d.y;
                gdir.y -= gt * t / d.y;
                camera_adjoint(gcam, gdir, gf, go, d, lw, right, up, f, l0, l1, l2, sx, sy);
            }
        } else {

            // The instance (the caller's matrices, as the forward saw them), its inverse, and the hit triangle in
            // mesh space.
            const float *mm = a.matrices + 12LL * inst;
            M3 A;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) A.a[r][c] = mm[4 * r + c];
            const M3 Ai = inverse(A);
            const int slot = inst - world * P;
            const int tri = __ldg(a.tri_of_local + __ldg(a.slot_tri_base + slot) + a.hit_triangle[pix]);
            const float3 v0 = xyz(__ldg(s.tris + 3LL * tri)), e1 = xyz(__ldg(s.tris + 3LL * tri + 1));
            const float3 e2 = xyz(__ldg(s.tris + 3LL * tri + 2));
            const float hu = a.hit_u[pix], hv = a.hit_v[pix];
            const float3 p = v0 + e1 * hu + e2 * hv;
            const float3 n = mul_t(Ai, cross(e1, e2));  // A^-T (e1 x e2)
            const float nd = dot(n, d);
            const float ln = sqrtf(dot(n, n));
            const float3 geo = n * (1.0f / ln);
            const float s_geo = dot(geo, d) > 0.0f ? -1.0f : 1.0f;

            M3 gA{};
            float3 gb = mk3(0.0f, 0.0f, 0.0f);
            float gt = 0.0f;

            // The normal: N = s m / |m|, m = A^-T n_s.
            if (gn.x != 0.0f || gn.y != 0.0f || gn.z != 0.0f) {
                bool smooth = false;
                float3 ns = cross(e1, e2), n0 = ns, n1 = ns, n2 = ns;
                if (s.attrs != nullptr) {
                    const float4 a0 = __ldg(s.attrs + 4LL * tri), a1 = __ldg(s.attrs + 4LL * tri + 1);
                    const float4 a2 = __ldg(s.attrs + 4LL * tri + 2), a3 = __ldg(s.attrs + 4LL * tri + 3);
                    if (__float_as_int(a3.w) & 1) {
                        n0 = xyz(a0);
                        n1 = xyz(a1);
                        n2 = xyz(a2);
                        const float3 blend = n0 * (1.0f - hu - hv) + n1 * hu + n2 * hv;
                        if (dot(blend, blend) > 1e-12f) {
                            ns = blend;
                            smooth = true;
                        }
                    }
                }
                const float3 m = mul_t(Ai, ns);
                const float lm = sqrtf(dot(m, m));
                const float3 mh = m * (1.0f / lm);
                const float sgn = smooth ? (dot(mh, geo * s_geo) < 0.0f ? -1.0f : 1.0f) : s_geo;
                const float3 gm = normalize_adjoint(mh, lm, gn * sgn);
                const float3 ai_gm = mul(Ai, gm);  // A^-1 gm
                add_outer(gA, m, ai_gm, -1.0f);     // through A^-T
                if (smooth) {
                    // Through the barycentrics: the point slides on the triangle as everything moves.
                    const float gu = dot(ai_gm, n1 - n0), gv = dot(ai_gm, n2 - n0);
                    const float e11 = dot(e1, e1), e22 = dot(e2, e2), e12 = dot(e1, e2);
                    const float det = e11 * e22 - e12 * e12;
                    const float3 a1 = (e1 * e22 - e2 * e12) * (1.0f / det);
                    const float3 a2 = (e2 * e11 - e1 * e12) * (1.0f / det);
                    const float3 gp = a1 * gu + a2 * gv;  // on the local point p = A^-1 (P - b)
                    const float3 gP = mul_t(Ai, gp);      // A^-T gp
                    gb = gb - gP;
                    add_outer(gA, gP, p, -1.0f);
                    go = go + gP;  // P = o + t d
                    gt += dot(gP, d);
                    gdir = gdir + gP * t;
                }
            }
            // The depth: D = t (d . f).
            gt += gd * df;
            gdir = gdir + f * (gd * t);
            gf = gf + d * (gd * t);
            // t = n . (A p + b - o) / (n . d).
            const float k = gt / nd;
            add_outer(gA, n, p, k);
            gb = gb + n * k;
            go = go - n * k;
            gdir = gdir - n * (k * t);
            camera_adjoint(gcam, gdir, gf, go, d, lw, right, up, f, l0, l1, l2, sx, sy);
            const float g[12] = {gA.a[0][0], gA.a[0][1], gA.a[0][2], gb.x, gA.a[1][0], gA.a[1][1], gA.a[1][2], gb.y,
                gA.a[2][0], gA.a[2][1], gA.a[2][2], gb.z};
            for (int e = 0; e < 12; ++e) ginst[e] = g[e];
            owner = inst;
        }
    }
    // Sums over the warp before any atomic: the camera's in one tree (a warp's pixels share the view), the
    // instances' one distinct instance at a time (a tile's warp sees few of them).
    const int lane = threadIdx.x & 31;
    const int entry = lane >> 1;  // the sum this lane holds after warp_sums12
    const bool adds = (lane & 1) == 0 && entry < 12;
    {
        const float v = warp_sums12(gcam, lane);
        if (adds && v != 0.0f) atomicAdd(cam_sum + entry, v);
    }
    for (unsigned pending = __ballot_sync(0xffffffffu, owner >= 0); pending != 0;) {
        const int inst_k = __shfl_sync(0xffffffffu, owner, __ffs(pending) - 1);
        const bool mine = owner == inst_k;
        pending &= ~__ballot_sync(0xffffffffu, mine);
        float *dst = shared_sums ? sums + 12 * (inst_k - world * P) : a.grad_matrices + 12LL * inst_k;
        float part[12];
        for (int e = 0; e < 12; ++e) part[e] = mine ? ginst[e] : 0.0f;
        const float v = warp_sums12(part, lane);
        if (adds && v != 0.0f) atomicAdd(dst + entry, v);
    }
    __syncthreads();
    if (shared_sums)
        for (int k = threadIdx.x; k < 12 * P; k += ADJ_THREADS) {
            const float v = sums[k];
            if (v != 0.0f) atomicAdd(a.grad_matrices + 12LL * world * P + k, v);
        }
    if (threadIdx.x < 12 && cam_sum[threadIdx.x] != 0.0f)
        atomicAdd(a.grad_cameras + 12LL * view + threadIdx.x, cam_sum[threadIdx.x]);
}

}  // namespace

cudaError_t launch_depth_normal_adjoint(const SceneParams &s, const AdjointArgs &a, cudaStream_t stream) {
    const int tiles_x = (a.width + ADJ_TILE - 1) / ADJ_TILE, tiles_y = (a.rows + ADJ_TILE - 1) / ADJ_TILE;
    const long long blocks = static_cast<long long>(tiles_x) * tiles_y * a.views;
    if (blocks == 0) return cudaSuccess;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    // Per-instance sums in shared memory for worlds of up to 1024 instances (48 KB), else straight to global.
    const bool shared_sums = s.per_world <= 1024;
    const size_t smem = sizeof(float) * ((shared_sums ? 12 * static_cast<size_t>(s.per_world) : 0) + 12);
    cudaError_t e = cudaFuncSetAttribute(depth_normal_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    depth_normal_adjoint_kernel<<<static_cast<unsigned>(blocks), ADJ_THREADS, smem, stream>>>(s, a, tiles_x,
        tiles_x * tiles_y, shared_sums);
    return cudaGetLastError();
}

}  // namespace ngb
