"""Differentiable depth and normal images.

    depth, normals = render_depth_normals(renderer, matrices, cameras, fov)
    loss = ((depth - target)[mask] ** 2).sum()
    loss.backward()            # -> matrices.grad, cameras.grad

matrices: (world_count, instances_per_world, 3, 4) world-from-mesh, float32 CUDA; cameras: (views, 3, 4)
camera-to-world, float32 CUDA. The forward renders with hit records on and keeps, per pixel, the centre ray's
(instance, triangle, barycentric) hit; the backward is one adjoint kernel (csrc/adjoint.cu) that holds
visibility fixed: each pixel's hit point moves with its instance and its ray moves with the camera, so the
gradient is that of a smooth function on every pixel away from silhouettes. Pixels whose ray hit no mesh
(sky, floor, spheres) carry no gradient.

pose_matrices builds the matrices from positions, quaternions and scales in torch, so gradients reach poses
through autograd: the quaternion is normalised first, as the pose compose does (quat_matrix,
src/cuda_backend.cu:165-172).
"""

from __future__ import annotations

import torch


class _DepthNormals(torch.autograd.Function):
    @staticmethod
    def forward(ctx, renderer, matrices, cameras, fov):
        m = matrices.detach().contiguous()
        c = cameras.detach().contiguous()
        renderer.set_instance_transforms(m)
        views, h, w = renderer.view_count, renderer.rows[1], renderer.width
        depth = torch.empty((views, h, w), dtype=torch.float32, device=m.device)
        normals = torch.empty((views, h, w, 3), dtype=torch.float32, device=m.device)
        hits = (torch.empty(depth.shape, dtype=torch.int32, device=depth.device),
                torch.empty(depth.shape, dtype=torch.int32, device=depth.device),
                torch.empty(depth.shape, dtype=torch.float32, device=depth.device),
                torch.empty(depth.shape, dtype=torch.float32, device=depth.device))
        # The render writes the hit records straight into the tensors saved for the backward; the renderer goes
        # back to not recording once the render is queued.
        renderer.record_hits(True, into=hits)
        try:
            renderer.render(c, fov, 1, rgb=False, depth=True, normals=True, into={"depth": depth, "normals": normals})
        finally:
            renderer.record_hits(False)
        ctx.renderer = renderer
        ctx.fov = float(fov)
        ctx.save_for_backward(m, c, depth, *hits)
        return depth, normals

    @staticmethod
    def backward(ctx, grad_depth, grad_normals):
        m, c, depth, *hits = ctx.saved_tensors
        gm = torch.zeros_like(m)
        gc = torch.zeros_like(c)
        gd = grad_depth.contiguous() if grad_depth is not None else torch.zeros_like(depth)
        gn = grad_normals.contiguous() if grad_normals is not None else None
        ctx.renderer.depth_normal_adjoint(m, c, ctx.fov, hits, depth, gd, gn, gm, gc)
        return None, gm, gc, None


def render_depth_normals(renderer, matrices, cameras, fov=1.0):
    """Depth (views, H, W) and normals (views, H, W, 3), differentiable in matrices and cameras."""
    return _DepthNormals.apply(renderer, matrices, cameras, fov)


class _PoseMatrices(torch.autograd.Function):
    """pose_matrices on float32 CUDA tensors of one shape: one kernel each way (ngb_pose_matrices and
    ngb_pose_matrices_grad) instead of the dozens of small element-wise kernels of the PyTorch form."""

    @staticmethod
    def forward(ctx, positions, quaternions, scales):
        import ctypes as C
        from ._lib import check, lib
        L = lib()
        out = torch.empty(positions.shape[:-1] + (3, 4), dtype=torch.float32, device=positions.device)
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        with torch.cuda.device(positions.device):
            stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            check(L.ngb_pose_matrices(ptr(positions), ptr(quaternions), ptr(scales), out.numel() // 12, ptr(out), stream))
        ctx.save_for_backward(quaternions, scales)
        return out

    @staticmethod
    def backward(ctx, grad):
        import ctypes as C
        from ._lib import check, lib
        L = lib()
        quaternions, scales = ctx.saved_tensors
        grad = grad.contiguous()
        lead = quaternions.shape[:-1]
        gp = torch.empty(lead + (3,), dtype=torch.float32, device=grad.device)
        gq = torch.empty(lead + (4,), dtype=torch.float32, device=grad.device)
        gs = torch.empty(lead + (3,), dtype=torch.float32, device=grad.device) if (
            scales is not None and ctx.needs_input_grad[2]) else None
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        with torch.cuda.device(grad.device):
            stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            check(L.ngb_pose_matrices_grad(ptr(quaternions), ptr(scales), grad.numel() // 12, ptr(grad), ptr(gp), ptr(gq),
                                           ptr(gs), stream))
        return gp, gq, gs


def quaternion_matrix(q):
    """Rotation matrices (..., 3, 3) of quaternions (..., 4) stored (x, y, z, w), normalised first."""
    q = q / torch.linalg.norm(q, dim=-1, keepdim=True)
    x, y, z, w = q.unbind(-1)
    return torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1).unflatten(-1, (3, 3))


def pose_matrices(positions, quaternions, scales=None):
    """3 x 4 matrices [R(q) diag(s) | p] of positions (..., 3), quaternions (..., 4) and scales (..., 3).
    Float32 CUDA tensors take the fused kernels (broadcast to one leading shape first); other tensors (CPU,
    float64 references) the PyTorch form below."""
    tensors = [t for t in (positions, quaternions, scales) if t is not None]
    if all(t.is_cuda and t.dtype == torch.float32 for t in tensors):
        lead = torch.broadcast_shapes(*[t.shape[:-1] for t in tensors])
        p = positions.expand(lead + (3,)).contiguous()
        q = quaternions.expand(lead + (4,)).contiguous()
        s = None if scales is None else scales.expand(lead + (3,)).contiguous()
        return _PoseMatrices.apply(p, q, s)
    r = quaternion_matrix(quaternions)
    if scales is not None:
        r = r * scales.unsqueeze(-2)
    return torch.cat([r, positions.unsqueeze(-1)], -1)
