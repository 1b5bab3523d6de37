"""The adjoint of the depth and normal images (csrc/adjoint.cu behind autodiff.render_depth_normals).

Two checks, both with visibility held fixed as the adjoint holds it:
  - against a float64 restatement in torch on the CPU (tests/adjoint_ref.py): the same pixels, the same
    recorded triangles, depth and normals written as smooth functions of the instance and camera matrices
    (ray-plane intersection, barycentric blend of vertex normals, the forward's facing choices) and
    differentiated by torch's autograd;
  - against central finite differences (h = 1e-3) of an L2 depth loss rendered end to end, on pixels at
    least 2 px from any object-ID change, with respect to instance positions and quaternions (through
    pose_matrices) and the camera position.
The bar: relative error of the gradient at most 1e-3.
"""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
from neraulgraphics_b200 import workloads

from adjoint_ref import reference_depth_normals, rel_err, silhouette_free

pytestmark = pytest.mark.gpu


def make(worlds=4, width=48, height=40, seed=3):
    wl = workloads.differentiable_worlds(worlds=worlds, width=width, height=height, seed=seed)
    d = wl.desc
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device="cuda:0")
    return wl, r


def test_adjoint_is_the_float64_reference(torch_cuda):
    torch = torch_cuda
    from neraulgraphics_b200.autodiff import render_depth_normals
    wl, r = make()
    mats = torch.from_numpy(wl.matrices).cuda().requires_grad_()
    cams = torch.from_numpy(wl.cameras).cuda().requires_grad_()
    depth, normals = render_depth_normals(r, mats, cams, wl.fov)
    assert bool(torch.isfinite(depth).any())
    gen = torch.Generator(device="cuda").manual_seed(5)
    gd = torch.randn(depth.shape, device="cuda", generator=gen)
    gn = torch.randn(normals.shape, device="cuda", generator=gen)
    finite = torch.isfinite(depth)
    loss = (torch.where(finite, depth, 0.0) * gd).sum() + (normals * gn).sum()
    loss.backward()
    # The same pixels and triangles in float64: the forward's hits, recorded again by the same render.
    hits = [torch.empty(depth.shape, dtype=dt, device="cuda") for dt in (torch.int32, torch.int32, torch.float32, torch.float32)]
    r.record_hits(True)
    r.render(cams.detach(), wl.fov, 1, rgb=False, depth=True, normals=True, zero_copy=True)
    r.copy_hits(*hits)
    r.record_hits(False)
    # The float64 reference runs on the CPU, from the host copies of the recorded hits.
    m64 = torch.from_numpy(wl.matrices).double().requires_grad_()
    c64 = torch.from_numpy(wl.cameras).double().requires_grad_()
    hits_cpu = [h.cpu() for h in hits]
    d64, n64 = reference_depth_normals(torch, wl.desc, m64, c64, hits_cpu, depth.detach().cpu(), wl.fov)
    mesh = hits_cpu[0] >= 0
    assert float(mesh.float().mean()) > 0.1
    # The reference reproduces the forward (visibility fixed, so the same values up to float32 rounding).
    fin = finite.cpu()
    assert float((d64.detach()[fin] - depth.detach().cpu()[fin].double()).abs().max()) < 1e-3
    ref = (d64 * gd.cpu().double()).sum() + (n64 * gn.cpu().double()).sum()
    gm, gc = torch.autograd.grad(ref, (m64, c64))
    assert bool(torch.isfinite(mats.grad).all()) and bool(torch.isfinite(cams.grad).all())
    assert bool(torch.isfinite(gm).all()) and bool(torch.isfinite(gc).all())
    em = rel_err(mats.grad.double().cpu().numpy(), gm.cpu().numpy())
    ec = rel_err(cams.grad.double().cpu().numpy(), gc.cpu().numpy())
    assert em <= 1e-3 and ec <= 1e-3, (em, ec)


def test_adjoint_matches_central_differences(torch_cuda):
    """An L2 depth loss against a target depth 0.5 nearer than the scene's own, so that every pixel's weight
    2 (D - T) is about 1 and a parameter's pixels add up instead of cancelling: the float32 rounding of the
    rendered depths (a few 1e-6 per pixel, over 2h) then stays far below the gradient it is compared with."""
    torch = torch_cuda
    from neraulgraphics_b200.autodiff import pose_matrices, render_depth_normals
    wl, r = make(worlds=2, width=64, height=48, seed=9)
    info = wl.info
    T = lambda a: torch.from_numpy(a).cuda()
    pos, quat, scale = T(info["positions"]), T(info["quaternions"]), T(info["scales"])
    cams = T(wl.cameras)
    with torch.no_grad():
        base = render_depth_normals(r, pose_matrices(pos, quat, scale), cams, wl.fov)[0].clone()
    ids = r.render(cams, wl.fov, 1, rgb=False, object_ids=True, zero_copy=True)["object_ids"].cpu().numpy()
    mask = T(silhouette_free(ids)) & torch.isfinite(base)
    target = torch.where(mask, base - 0.5, 0.0)

    def loss_of(p, q, c):
        depth = render_depth_normals(r, pose_matrices(p, q, scale), c, wl.fov)[0]
        return (torch.where(mask, depth - target, 0.0) ** 2).sum()

    p, q, c = pos.clone().requires_grad_(), quat.clone().requires_grad_(), cams.clone().requires_grad_()
    loss_of(p, q, c).backward()
    h = 1e-3
    got, fd = [], []
    with torch.no_grad():
        for w in range(2):
            for i in range(12):
                for which, k in [(0, j) for j in range(3)] + [(1, j) for j in range(4)]:
                    arr = pos if which == 0 else quat
                    plus, minus = arr.clone(), arr.clone()
                    plus[w, i, k] += h
                    minus[w, i, k] -= h
                    lp = loss_of(plus, quat, cams) if which == 0 else loss_of(pos, plus, cams)
                    lm = loss_of(minus, quat, cams) if which == 0 else loss_of(pos, minus, cams)
                    fd.append(float(lp - lm) / (2 * h))
                    got.append(float((p.grad if which == 0 else q.grad)[w, i, k]))
            for k in range(3):  # the camera position: the matrix's last column
                plus, minus = cams.clone(), cams.clone()
                plus[w, k, 3] += h
                minus[w, k, 3] -= h
                fd.append(float(loss_of(pos, quat, plus) - loss_of(pos, quat, minus)) / (2 * h))
                got.append(float(c.grad[w, k, 3]))
    got, fd = np.array(got), np.array(fd)
    assert (np.abs(fd) > 1.0).sum() >= 20  # most instances are in view and move the loss
    assert rel_err(got, fd) <= 1e-3, (rel_err(got, fd), np.c_[got, fd][np.argsort(-np.abs(got - fd))[:8]])


def test_fused_pose_matrices_match_the_torch_form(torch_cuda):
    """pose_matrices on float32 CUDA tensors (the fused forward and gradient kernels) against its PyTorch form
    in float64: matrices within float32 rounding, gradients of a random linear loss within 1e-5 relative, for
    unnormalised quaternions, uneven scales and a broadcast scale."""
    torch = torch_cuda
    from neraulgraphics_b200.autodiff import pose_matrices
    gen = torch.Generator(device="cpu").manual_seed(3)
    p = torch.randn(7, 33, 3, generator=gen)
    q = torch.randn(7, 33, 4, generator=gen) * 3.0
    s = torch.rand(7, 33, 3, generator=gen) + 0.5
    g = torch.randn(7, 33, 3, 4, generator=gen)
    for scales in (s, s[0], None):
        args32 = [t.cuda().requires_grad_() for t in (p, q)] + ([scales.cuda().requires_grad_()] if scales is not None else [])
        args64 = [t.double().requires_grad_() for t in (p, q)] + ([scales.double().requires_grad_()] if scales is not None else [])
        m32 = pose_matrices(*args32) if scales is not None else pose_matrices(*args32, None)
        m64 = pose_matrices(*args64) if scales is not None else pose_matrices(*args64, None)
        assert m32.shape == (7, 33, 3, 4)
        assert float((m32.detach().cpu().double() - m64.detach()).abs().max()) < 2e-6 * (float(m64.detach().abs().max()) + 1)
        (m32 * g.cuda()).sum().backward()
        (m64 * g.double()).sum().backward()
        for a, b in zip(args32, args64):
            err = float((a.grad.cpu().double() - b.grad).abs().max())
            assert err <= 1e-5 * (float(b.grad.abs().max()) + 1e-3), err
