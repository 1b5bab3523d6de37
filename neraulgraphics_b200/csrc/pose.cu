// Instance matrices from poses, [R(q) diag(s) | p] with q normalised first, and their gradient: one thread per
// pose, one launch each way, for the differentiable path (autodiff.pose_matrices on float32 CUDA tensors). The
// forward is the float arithmetic of that function's PyTorch form, expression by expression; the backward is
// the transposed derivative of the same expressions.
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/ngb.h"

namespace ngb {
void set_global_error(const std::string &message);  // renderer.cpp: what ngb_last_error(NULL) returns
}

namespace {

int fail(int status, const std::string &message) {
    ngb::set_global_error(message);
    return status;
}

__device__ __forceinline__ void rotation(const float *qn, float *r) {
    const float x = qn[0], y = qn[1], z = qn[2], w = qn[3];
    r[0] = 1.0f - 2.0f * (y * y + z * z);
    r[1] = 2.0f * (x * y - z * w);
    r[2] = 2.0f * (x * z + y * w);
    r[3] = 2.0f * (x * y + z * w);
    r[4] = 1.0f - 2.0f * (x * x + z * z);
    r[5] = 2.0f * (y * z - x * w);
    r[6] = 2.0f * (x * z - y * w);
    r[7] = 2.0f * (y * z + x * w);
    r[8] = 1.0f - 2.0f * (x * x + y * y);
}

// The quaternion over its norm, and the norm.
__device__ __forceinline__ float normalised(const float *q, long long i, float *qn) {
    float v[4];
    for (int k = 0; k < 4; ++k) v[k] = __ldg(q + 4 * i + k);
    const float n = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
    for (int k = 0; k < 4; ++k) qn[k] = v[k] / n;
    return n;
}

__global__ void pose_kernel(const float *p, const float *q, const float *s, long long count, float *m) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    float qn[4], r[9];
    normalised(q, i, qn);
    rotation(qn, r);
    float *out = m + 12 * i;
    for (int row = 0; row < 3; ++row) {
        for (int col = 0; col < 3; ++col) out[4 * row + col] = s ? r[3 * row + col] * __ldg(s + 3 * i + col) : r[3 * row + col];
        out[4 * row + 3] = __ldg(p + 3 * i + row);
    }
}

// d(loss)/d(p, q, s) from d(loss)/d(matrix) g: g's last column for p; per column j, sum_i g[i][j] R[i][j] for s;
// and through R = R(q / |q|) for q.
__global__ void pose_grad_kernel(const float *q, const float *s, long long count, const float *g, float *gp, float *gq,
    float *gs) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    float qn[4], r[9], gr[9];
    const float n = normalised(q, i, qn);
    rotation(qn, r);
    const float *gi = g + 12 * i;
    for (int row = 0; row < 3; ++row) {
        gp[3 * i + row] = __ldg(gi + 4 * row + 3);
        for (int col = 0; col < 3; ++col) {
            const float sc = s ? __ldg(s + 3 * i + col) : 1.0f;
            gr[3 * row + col] = __ldg(gi + 4 * row + col) * sc;
        }
    }
    if (gs)
        for (int col = 0; col < 3; ++col)
            gs[3 * i + col] = __ldg(gi + col) * r[col] + __ldg(gi + 4 + col) * r[3 + col] + __ldg(gi + 8 + col) * r[6 + col];
    const float x = qn[0], y = qn[1], z = qn[2], w = qn[3];
    // dR/dx, dR/dy, dR/dz, dR/dw contracted with gr.
    const float dx = 2.0f * (y * (gr[1] + gr[3]) + z * (gr[2] + gr[6]) + w * (gr[7] - gr[5])) - 4.0f * x * (gr[4] + gr[8]);
    const float dy = 2.0f * (x * (gr[1] + gr[3]) + w * (gr[2] - gr[6]) + z * (gr[5] + gr[7])) - 4.0f * y * (gr[0] + gr[8]);
    const float dz = 2.0f * (w * (gr[3] - gr[1]) + x * (gr[2] + gr[6]) + y * (gr[5] + gr[7])) - 4.0f * z * (gr[0] + gr[4]);
    const float dw = 2.0f * (z * (gr[3] - gr[1]) + y * (gr[2] - gr[6]) + x * (gr[7] - gr[5]));
    // Through qn = q / n: (g - qn (qn . g)) / n.
    const float dot = x * dx + y * dy + z * dz + w * dw;
    gq[4 * i] = (dx - x * dot) / n;
    gq[4 * i + 1] = (dy - y * dot) / n;
    gq[4 * i + 2] = (dz - z * dot) / n;
    gq[4 * i + 3] = (dw - w * dot) / n;
}

unsigned blocks_of(long long count) { return static_cast<unsigned>((count + 255) / 256); }

}  // namespace

extern "C" int ngb_pose_matrices(const float *positions, const float *quaternions, const float *scales, int64_t count,
    float *matrices, void *stream) {
    if (count < 0) return fail(NGB_INVALID_ARGUMENT, "count must be 0 or more");
    if (count == 0) return NGB_OK;
    if (!positions || !quaternions || !matrices)
        return fail(NGB_INVALID_ARGUMENT, "positions, quaternions and matrices must not be null");
    pose_kernel<<<blocks_of(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(positions, quaternions, scales, count,
        matrices);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NGB_OK : fail(NGB_CUDA_ERROR, std::string("pose kernel: ") + cudaGetErrorString(e));
}

extern "C" int ngb_pose_matrices_grad(const float *quaternions, const float *scales, int64_t count,
    const float *grad_matrices, float *grad_positions, float *grad_quaternions, float *grad_scales, void *stream) {
    if (count < 0) return fail(NGB_INVALID_ARGUMENT, "count must be 0 or more");
    if (count == 0) return NGB_OK;
    if (!quaternions || !grad_matrices || !grad_positions || !grad_quaternions)
        return fail(NGB_INVALID_ARGUMENT, "quaternions, grad_matrices, grad_positions and grad_quaternions must not be null");
    if (grad_scales && !scales) return fail(NGB_INVALID_ARGUMENT, "grad_scales needs scales");
    pose_grad_kernel<<<blocks_of(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(quaternions, scales, count,
        grad_matrices, grad_positions, grad_quaternions, grad_scales);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NGB_OK : fail(NGB_CUDA_ERROR, std::string("pose gradient kernel: ") + cudaGetErrorString(e));
}
