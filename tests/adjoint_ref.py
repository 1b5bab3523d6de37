"""Test helpers for the adjoint checks: a float64 restatement of the depth and normal images as smooth
functions of the instance and camera matrices (visibility held fixed at the recorded hits), runnable on CPU
tensors, and the silhouette mask of the finite-difference checks."""

import numpy as np


def rel_err(got, want):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30))


def reference_depth_normals(torch, desc, mats, cams, hits, depth, fov, first_instance=0):
    """float64 depth and normals of the recorded hits as functions of mats (W, N, 3, 4) and cams (V, 3, 4), on the
    device of the hit tensors (the CPU for the float64 reference). desc: the scene (its view_count, height, width,
    per_world, instances, meshes and floor); first_instance: the global index of mats' first instance, when the
    hits are a slice of a larger batch's."""
    d = desc
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
        g = inst[m].long() - first_instance
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
