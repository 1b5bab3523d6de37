"""The adjoint of the depth and normal images (csrc/adjoint.cu behind autodiff.render_depth_normals).

Two checks, both with visibility held fixed as the adjoint holds it:
  - against a float64 restatement in torch: the same pixels, the same recorded triangles, depth and normals
    written as smooth functions of the instance and camera matrices (ray-plane intersection, barycentric
    blend of vertex normals, the forward's facing choices) and differentiated by torch's autograd;
  - against central finite differences (h = 1e-3) of an L2 depth loss rendered end to end, on pixels at
    least 2 px from any object-ID change, with respect to instance positions and quaternions (through
    pose_matrices) and the camera position.
The bar: relative error of the gradient at most 1e-3.
"""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu


def make(worlds=4, width=48, height=40, seed=3):
    wl = workloads.differentiable_worlds(worlds=worlds, width=width, height=height, seed=seed)
    d = wl.desc
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device="cuda:0")
    return wl, r


def rel_err(got, want):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30))


def reference_depth_normals(torch, wl, mats, cams, hits, depth, fov):
    """float64 depth and normals of the recorded hits as functions of mats (W, N, 3, 4) and cams (V, 3, 4)."""
    d = wl.desc
    V, H, W = d.view_count, d.height, d.width
    inst, tri, hu, hv = (h.reshape(-1) for h in hits)
    dep = depth.reshape(-1)
    pix = torch.arange(V * H * W, device=inst.device)
    view, rem = pix // (H * W), pix % (H * W)
    y, x = (rem // W).double(), (rem % W).double()
    cm = cams[view]                                                 # (P, 3, 4)
    c0, c1, c2, o = cm[..., 0], cm[..., 1], cm[..., 2], cm[..., 3]
    unit = lambda v: v / torch.linalg.norm(v, dim=-1, keepdim=True)
    right, up, f = unit(c0), unit(c1), unit(-c2)
    fs = np.tan(fov * 0.5)
    sx = ((2.0 * (x + 0.5) / W - 1.0) * fs * (W / H)).unsqueeze(-1)
    sy = (-(2.0 * (y + 0.5) / H - 1.0) * fs).unsqueeze(-1)
    dr = unit(right * sx + up * sy + f)
    depth_out = torch.zeros(V * H * W, dtype=torch.float64, device=inst.device)
    normal_out = torch.zeros(V * H * W, 3, dtype=torch.float64, device=inst.device)
    # Mesh hits: the recorded triangle, moving with its instance.
    m = inst >= 0
    if bool(m.any()):
        P = d.per_world
        g = inst[m].long()
        A, b = mats.reshape(-1, 3, 4)[g, :, :3], mats.reshape(-1, 3, 4)[g, :, 3]
        slot = (g % P).cpu().numpy()
        mesh_of = np.array([d.instances[i].mesh for i in range(P)])[slot]
        t_idx = tri[m].cpu().numpy()
        v0 = np.zeros((len(slot), 3)); e1 = np.zeros_like(v0); e2 = np.zeros_like(v0)
        n0 = np.zeros_like(v0); n1 = np.zeros_like(v0); n2 = np.zeros_like(v0); smooth = np.zeros(len(slot), bool)
        for k, mesh in enumerate(d.meshes):
            sel = mesh_of == k
            idx = mesh.triangles[t_idx[sel]]
            vv = mesh.vertices.astype(np.float64)
            v0[sel] = vv[idx[:, 0]]
            e1[sel] = vv[idx[:, 1]] - vv[idx[:, 0]]
            e2[sel] = vv[idx[:, 2]] - vv[idx[:, 0]]
            if mesh.normals is not None:
                nn = mesh.normals.astype(np.float64)
                n0[sel], n1[sel], n2[sel] = nn[idx[:, 0]], nn[idx[:, 1]], nn[idx[:, 2]]
                smooth[sel] = True
        T = lambda a: torch.from_numpy(a).to(inst.device)
        v0, e1, e2, n0, n1, n2, smooth = map(T, (v0, e1, e2, n0, n1, n2, smooth))
        om, dm, fm = o[m], dr[m], f[m]
        V0 = torch.einsum("pij,pj->pi", A, v0) + b
        E1, E2 = torch.einsum("pij,pj->pi", A, e1), torch.einsum("pij,pj->pi", A, e2)
        nw = torch.cross(E1, E2, dim=-1)
        t = ((V0 - om) * nw).sum(-1) / (dm * nw).sum(-1)
        Pw = om + t.unsqueeze(-1) * dm
        # Barycentrics of the moving point (dual basis of E1, E2 in the plane).
        q = Pw - V0
        e11, e22, e12 = (E1 * E1).sum(-1), (E2 * E2).sum(-1), (E1 * E2).sum(-1)
        det = e11 * e22 - e12 * e12
        u = (e22 * (q * E1).sum(-1) - e12 * (q * E2).sum(-1)) / det
        v = (e11 * (q * E2).sum(-1) - e12 * (q * E1).sum(-1)) / det
        Ait = torch.linalg.inv(A).transpose(-1, -2)
        geo = unit(torch.einsum("pij,pj->pi", Ait, torch.cross(e1, e2, dim=-1)))
        s_geo = torch.where((geo.detach() * dm.detach()).sum(-1, keepdim=True) > 0, -1.0, 1.0)
        geo = geo * s_geo
        ns = n0 * (1 - u - v).unsqueeze(-1) + n1 * u.unsqueeze(-1) + n2 * v.unsqueeze(-1)
        # Rows without vertex normals blend zeros: give them the geometric normal, so that the branch
        # torch.where does not take stays finite (its gradient would be 0 * NaN otherwise).
        ns = torch.where(smooth.unsqueeze(-1), ns, torch.cross(e1, e2, dim=-1))
        sm = unit(torch.einsum("pij,pj->pi", Ait, ns))
        s_sm = torch.where((sm.detach() * geo.detach()).sum(-1, keepdim=True) < 0, -1.0, 1.0)
        normal = torch.where(smooth.unsqueeze(-1), sm * s_sm, geo)
        depth_out = depth_out.index_put((m.nonzero()[:, 0],), t * (dm * fm).sum(-1))
        normal_out = normal_out.index_put((m.nonzero()[:, 0],), normal)
    # Floor hits: the plane y = floor.y, moving with nothing but the camera.
    fl = (inst < 0) & torch.isfinite(dep)
    if bool(fl.any()):
        t = (d.floor.y - o[fl][:, 1]) / dr[fl][:, 1]
        depth_out = depth_out.index_put((fl.nonzero()[:, 0],), t * (dr[fl] * f[fl]).sum(-1))
    return depth_out.reshape(V, H, W), normal_out.reshape(V, H, W, 3)


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
    m64 = torch.from_numpy(wl.matrices).cuda().double().requires_grad_()
    c64 = torch.from_numpy(wl.cameras).cuda().double().requires_grad_()
    d64, n64 = reference_depth_normals(torch, wl, m64, c64, hits, depth.detach(), wl.fov)
    mesh = hits[0] >= 0
    assert float(mesh.float().mean()) > 0.1
    # The reference reproduces the forward (visibility fixed, so the same values up to float32 rounding).
    assert float((d64.detach()[finite] - depth.detach()[finite].double()).abs().max()) < 1e-3
    ref = (d64 * gd.double()).sum() + (n64 * gn.double()).sum()
    gm, gc = torch.autograd.grad(ref, (m64, c64))
    assert bool(torch.isfinite(mats.grad).all()) and bool(torch.isfinite(cams.grad).all())
    assert bool(torch.isfinite(gm).all()) and bool(torch.isfinite(gc).all())
    em = rel_err(mats.grad.double().cpu().numpy(), gm.cpu().numpy())
    ec = rel_err(cams.grad.double().cpu().numpy(), gc.cpu().numpy())
    assert em <= 1e-3 and ec <= 1e-3, (em, ec)


def silhouette_free(ids, margin=2):
    """Pixels at least margin px (Chebyshev) from any change of object ID between 4-neighbours."""
    edge = np.zeros(ids.shape, bool)
    edge[:, 1:, :] |= ids[:, 1:, :] != ids[:, :-1, :]
    edge[:, :-1, :] |= ids[:, 1:, :] != ids[:, :-1, :]
    edge[:, :, 1:] |= ids[:, :, 1:] != ids[:, :, :-1]
    edge[:, :, :-1] |= ids[:, :, 1:] != ids[:, :, :-1]
    grown = edge.copy()
    H, W = ids.shape[1:]
    for dy in range(-margin, margin + 1):
        for dx in range(-margin, margin + 1):
            sh = np.zeros_like(edge)
            sh[:, max(dy, 0):H + min(dy, 0), max(dx, 0):W + min(dx, 0)] = \
                edge[:, max(-dy, 0):H + min(-dy, 0), max(-dx, 0):W + min(-dx, 0)]
            grown |= sh
    return ~grown


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
