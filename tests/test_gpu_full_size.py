"""Parity at the full sizes the path is measured at, with the product's default kernels.

- 4096 worlds x 20 bodies at 64x64 (RGB, depth, object IDs): every world against the oracle, the trees of all
  81,920 instances bit-exact, and the tile kernels against the persistent kernel (which walks the world trees in
  the reference's order) on every pixel;
- 2048 worlds of uneven sizes (1 to 200 instances of six meshes up to 20,480 triangles, 32/64/128 px) in one
  renderer: a stratified sample of worlds (every resolution, instance counts from the least to the most)
  against the oracle, world by world;
- one world of 100,000 instances at 1280x720 with a 64 x 2048 LiDAR sweep against the oracle;
- 1024 worlds at 128x128 (depth and normals) with the L2 depth loss against a target rendered from perturbed
  poses: the adjoint's gradient on a sample of worlds against a float64 CPU restatement, and against central
  differences (h = 1e-3) of a per-world float64 loss.

Pixels whose two nearest hits lie within 1e-6 relative t (the oracle flags them) are exempt from the bit-exact
comparison, since the tile kernels visit a world's instances in their own order; every test prints their count
and bounds it. The reference's own bound for two valid trees of one scene is 1 pixel in 2000 with a differing
object ID (tests/test_batch.cpp:335-374 in the reference); the near ties here must stay below 1 in 10,000.
"""

import types

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
from neraulgraphics_b200 import workloads

from adjoint_ref import reference_depth_normals, rel_err, silhouette_free

pytestmark = pytest.mark.gpu
TIE_BOUND = 1e-4  # near-tie pixels, as a fraction of the pixels compared


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def compare(got, want, ties, what):
    """Bit-exact IDs and depth (and normals when given), RGB within one level, off the near-tie pixels; returns
    (compared pixels, near-tie pixels, RGB pixels one level off)."""
    aov_ok = (ties & O.TIE_AOV_INSTANCE) == 0
    rgb_ok = (ties & O.TIE_RGB_INSTANCE) == 0
    assert np.array_equal(got["object_ids"][aov_ok], want["object_ids"][aov_ok]), what + ": object IDs"
    assert np.array_equal(bits(got["depth"][aov_ok]), bits(want["depth"][aov_ok])), what + ": depth"
    if "normals" in want:
        assert np.array_equal(bits(got["normals"][aov_ok]), bits(want["normals"][aov_ok])), what + ": normals"
    off = np.abs(got["rgb"].astype(int) - want["rgb"].astype(int)).max(-1)[rgb_ok]
    assert off.max(initial=0) <= 1, f"{what}: RGB off by {off.max()} levels at {(off > 1).sum()} pixels"
    return ties.size, int((ties != 0).sum()), int((off > 0).sum())


def test_body_worlds_at_4096_worlds(torch_cuda):
    wl = workloads.body_worlds()
    d = wl.desc
    assert d.world_count == 4096 and d.per_world == 20 and (d.width, d.height) == (64, 64)
    poses = workloads.random_walk(wl.poses, 2, seed=3)[-1]
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device="cuda:0")
    o = O.Oracle(d)
    for x in (r, o):
        x.bind_bodies(**wl.binding)
        x.set_body_poses(poses)
    got_tree, want_tree = r.inspect_tlas(), o.tlas()
    for k in ("keys", "sorted_ids", "roots"):
        assert np.array_equal(got_tree[k], want_tree[k]), k
    assert np.array_equal(got_tree["nodes"][:, [3, 7]], want_tree["nodes"][:, [3, 7]])
    assert np.array_equal(got_tree["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32),
                          want_tree["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32))
    assert np.array_equal(bits(got_tree["matrices"]), bits(want_tree["matrices"]))
    got = r.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=1)
    want = o.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=1, ties=True)
    assert (want["object_ids"] >= ng.OBJECT_INSTANCE).mean() > 0.05
    n, ties, rgb1 = compare(got, want, want["ties"], "4096 worlds")
    print(f"\n4096 x 64x64: {n} pixels, near ties {ties} ({ties / n:.2e}), RGB one level off {rgb1}")
    assert ties <= TIE_BOUND * n
    # The persistent kernel walks each world's tree in the reference's order: the tile kernels' images must be
    # its images on every pixel but the near ties.
    r.set_tuning(kernel=2)
    walk = r.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=1)
    differ = (walk["object_ids"] != got["object_ids"]) | (bits(walk["depth"]) != bits(got["depth"])) | \
        (walk["rgb"] != got["rgb"]).any(-1)
    print(f"tile kernels vs the persistent kernel: {int(differ.sum())} pixels differ")
    assert not (differ & (want["ties"] == 0)).any()


def test_uneven_worlds_at_2048_worlds(torch_cuda):
    wl = workloads.uneven_worlds()
    worlds = wl["worlds"]
    assert len(worlds) == 2048
    mats = workloads.walk_uneven(wl, 1, seed=2)[0]
    u = ng.UnevenBatchRenderer(worlds, lights=wl["lights"], floor=wl["floor"], meshes=wl["meshes"], device="cuda:0")
    u.set_instance_transforms(mats)
    got = u.render(wl["cameras"], wl["fov"], 1, rgb=True, depth=True, object_ids=True, frame=3)
    # A stratified sample: per resolution, 48 worlds evenly spaced in instance count, least and most included.
    counts, res = wl["counts"], wl["resolutions"]
    sample = []
    for size in (32, 64, 128):
        of = np.nonzero(res == size)[0]
        by_count = of[np.argsort(counts[of], kind="stable")]
        sample += list(by_count[np.linspace(0, len(by_count) - 1, 48).round().astype(int)])
    sample = sorted(set(int(w) for w in sample))
    assert counts[sample].min() <= 3 and counts[sample].max() >= 198
    first = u.instance_first
    total = ties_total = rgb1_total = 0
    for w in sample:
        width, height, insts = worlds[w]
        desc = ng.SceneDesc(width, height, 1, 1, [], wl["lights"], wl["floor"], wl["meshes"], insts)
        o = O.Oracle(desc)
        o.set_instance_transforms(mats[first[w]:first[w + 1]].reshape(1, len(insts), 3, 4))
        want = o.render(wl["cameras"][w:w + 1], wl["fov"], 1, rgb=True, depth=True, object_ids=True, frame=3, ties=True)
        mine = {k: u.image(v, w)[None] for k, v in got.items()}
        n, ties, rgb1 = compare(mine, want, want["ties"], f"world {w} ({len(insts)} instances, {width}px)")
        total, ties_total, rgb1_total = total + n, ties_total + ties, rgb1_total + rgb1
    print(f"\nuneven 2048 worlds, {len(sample)} sampled: {total} pixels, near ties {ties_total} "
          f"({ties_total / total:.2e}), RGB one level off {rgb1_total}")
    assert ties_total <= TIE_BOUND * total


def test_large_world_at_100000_instances(torch_cuda):
    wl = workloads.large_world()
    d = wl.desc
    assert d.per_world == 100_000 and (d.width, d.height) == (1280, 720)
    r = ng.BatchRenderer(d.width, d.height, 1, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances, device="cuda:0")
    o = O.Oracle(d)
    for x in (r, o):
        x.set_instance_transforms(wl.matrices[0])
    got_tree, want_tree = r.inspect_tlas(), o.tlas()
    for k in ("keys", "sorted_ids", "roots"):
        assert np.array_equal(got_tree[k], want_tree[k]), k
    got = r.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    want = o.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, ties=True)
    assert (want["object_ids"] >= ng.OBJECT_INSTANCE).mean() > 0.5
    n, ties, rgb1 = compare(got, want, want["ties"], "1280x720, 100,000 instances")
    print(f"\nlarge world: {n} pixels, near ties {ties} ({ties / n:.2e}), RGB one level off {rgb1}")
    assert ties <= TIE_BOUND * n
    lidar = wl.info["lidar"]
    hits = r.cast_rays(lidar["origins"], lidar["directions"], lidar["max_distance"])
    exp = o.cast_rays(lidar["origins"], lidar["directions"], lidar["max_distance"])
    assert (exp["object_id"] >= ng.OBJECT_INSTANCE).mean() > 0.5
    for k in ("object_id", "distance", "normal"):
        assert np.array_equal(bits(hits[k]), bits(exp[k])), k


def test_differentiable_worlds_at_1024_worlds(torch_cuda):
    torch = torch_cuda
    from neraulgraphics_b200.autodiff import pose_matrices, render_depth_normals
    wl = workloads.differentiable_worlds()
    d, info = wl.desc, wl.info
    assert d.world_count == 1024 and (d.width, d.height) == (128, 128)
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device="cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    scale = T(info["scales"])
    cams = T(wl.cameras)
    with torch.no_grad():
        target = render_depth_normals(r, pose_matrices(T(info["target_positions"]), T(info["target_quaternions"]),
                                                       scale), cams, wl.fov)[0].clone()
    # The loss of the differentiable form: L2 of the depth against the target, where both are finite.
    mats = pose_matrices(T(info["positions"]), T(info["quaternions"]), scale).detach().requires_grad_()
    cam = cams.clone().requires_grad_()
    depth, _ = render_depth_normals(r, mats, cam, wl.fov)
    both = torch.isfinite(depth.detach()) & torch.isfinite(target)
    loss = (torch.where(both, depth - target, 0.0) ** 2).sum()
    loss.backward()
    hits = [torch.empty(depth.shape, dtype=dt, device="cuda") for dt in (torch.int32, torch.int32, torch.float32, torch.float32)]
    r.record_hits(True)
    r.render(cam.detach(), wl.fov, 1, rgb=False, depth=True, normals=True, zero_copy=True)
    r.copy_hits(*hits)
    r.record_hits(False)
    weight = torch.where(both, 2.0 * (depth.detach() - target), 0.0).cpu().double()
    P = d.per_world
    sample = [0, 1, 137, 511, 512, 777, 1022, 1023]
    worst = 0.0
    for w in sample:
        one = types.SimpleNamespace(view_count=1, height=d.height, width=d.width, per_world=P, instances=d.instances,
                                    meshes=d.meshes, floor=d.floor)
        m64 = torch.from_numpy(mats.detach()[w:w + 1].cpu().numpy()).double().requires_grad_()
        c64 = torch.from_numpy(wl.cameras[w:w + 1]).double().requires_grad_()
        h = [x[w:w + 1].cpu() for x in hits]
        d64, _ = reference_depth_normals(torch, one, m64, c64, h, depth.detach()[w:w + 1].cpu(), wl.fov,
                                         first_instance=w * P)
        gm, gc = torch.autograd.grad((d64 * weight[w:w + 1]).sum(), (m64, c64))
        em = rel_err(mats.grad[w:w + 1].double().cpu().numpy(), gm.numpy())
        ec = rel_err(cam.grad[w:w + 1].double().cpu().numpy(), gc.numpy())
        worst = max(worst, em, ec)
        assert em <= 1e-3 and ec <= 1e-3, (w, em, ec)
    print(f"\n1024 x 128x128: gradient vs float64 CPU on {len(sample)} worlds, worst relative error {worst:.2e}")

    # Central differences of a per-world float64 loss, conditioned as test_gpu_adjoint's (target 0.5 nearer on
    # pixels at least 2 px from a silhouette), through pose_matrices, for two worlds of the full batch.
    pos, quat = T(info["positions"]), T(info["quaternions"])
    with torch.no_grad():
        base = render_depth_normals(r, pose_matrices(pos, quat, scale), cams, wl.fov)[0].clone()
    ids = r.render(cams, wl.fov, 1, rgb=False, object_ids=True, zero_copy=True)["object_ids"].cpu().numpy()
    fd_worlds = [5, 900]
    mask = T(silhouette_free(ids)) & torch.isfinite(base)
    near = torch.where(mask, base - 0.5, 0.0)

    def world_losses(p, q, c):
        dep = render_depth_normals(r, pose_matrices(p, q, scale), c, wl.fov)[0]
        return [float((torch.where(mask[w], dep[w] - near[w], 0.0).double() ** 2).sum()) for w in fd_worlds]

    p, q, c = pos.clone().requires_grad_(), quat.clone().requires_grad_(), cams.clone().requires_grad_()
    dep = render_depth_normals(r, pose_matrices(p, q, scale), c, wl.fov)[0]
    sum(((torch.where(mask[w], dep[w] - near[w], 0.0)) ** 2).sum() for w in fd_worlds).backward()
    step = 1e-3
    got, fd = [], []
    with torch.no_grad():
        for j, w in enumerate(fd_worlds):
            for i in range(P):
                for which, k in [(0, a) for a in range(3)] + [(1, a) for a in range(4)]:
                    arr = pos if which == 0 else quat
                    plus, minus = arr.clone(), arr.clone()
                    plus[w, i, k] += step
                    minus[w, i, k] -= step
                    lp = world_losses(plus, quat, cams) if which == 0 else world_losses(pos, plus, cams)
                    lm = world_losses(minus, quat, cams) if which == 0 else world_losses(pos, minus, cams)
                    fd.append((lp[j] - lm[j]) / (2 * step))
                    got.append(float((p.grad if which == 0 else q.grad)[w, i, k]))
            for k in range(3):
                plus, minus = cams.clone(), cams.clone()
                plus[w, k, 3] += step
                minus[w, k, 3] -= step
                fd.append((world_losses(pos, quat, plus)[j] - world_losses(pos, quat, minus)[j]) / (2 * step))
                got.append(float(c.grad[w, k, 3]))
    got, fd = np.array(got), np.array(fd)
    err = rel_err(got, fd)
    print(f"central differences on worlds {fd_worlds} of 1024: {len(got)} parameters, relative error {err:.2e}")
    assert (np.abs(fd) > 1.0).sum() >= 20
    assert err <= 1e-3, (err, np.c_[got, fd][np.argsort(-np.abs(got - fd))[:8]])
