"""GPU parity tests: the CUDA path, through the C ABI, against the oracle and the reference's own outputs.

The bar: tree keys, sorted orders, links and roots bit-exact; object IDs, hit triangles, depth and normals
bit-exact against the oracle on the same trees (and against the reference except where the two nearest hits
of a ray lie within 1e-6 relative t, which the oracle flags); RGB within one uint8 level (CUDA's sinf, cosf
and powf are within a few ulp of the host's).
"""

import os

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
import scenes
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ALL = dict(rgb=True, depth=True, normals=True, object_ids=True)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def product(desc):
    return ng.BatchRenderer(desc.width, desc.height, desc.world_count, desc.cameras_per_world, desc.spheres,
                            desc.lights, desc.floor, desc.meshes, desc.instances, device="cuda:0")


def assert_same_images(got, want, rgb_tol=1, ties=None):
    """Bit-exact IDs, depth and normals, RGB within rgb_tol levels. ties (the oracle's per-pixel flags), when
    given, exempts the pixels whose ray has two objects within 1e-6 relative t: the tile kernel visits a world's
    instances in another order than the world tree does, and which of two such hits it keeps may differ."""
    aov_ok = np.ones(got[next(iter(got))].shape[:3], bool) if ties is None else (ties & O.TIE_AOV_INSTANCE) == 0
    rgb_ok = aov_ok if ties is None else (ties & O.TIE_RGB_INSTANCE) == 0
    for k in ("object_ids",):
        if k in want:
            assert np.array_equal(got[k][aov_ok], want[k][aov_ok]), k
    for k in ("depth", "normals"):
        if k in want:
            assert np.array_equal(bits(got[k][aov_ok]), bits(want[k][aov_ok])), k
    if "rgb" in want:
        d = np.abs(got["rgb"].astype(int) - want["rgb"].astype(int)).max(-1)[rgb_ok]
        assert d.max(initial=0) <= rgb_tol, f"rgb differs by up to {d.max()} levels at {(d > rgb_tol).sum()} pixels"


def oracle_ties(desc, cameras, fov=1.0, matrices=None, binding=None, poses=None, frame=0, ambient=None):
    """The oracle's near-tie flags for these views."""
    o = O.Oracle(desc)
    if matrices is not None:
        o.set_instance_transforms(matrices)
    else:
        o.bind_bodies(**binding)
        o.set_body_poses(poses)
    if ambient is not None:
        o.set_ambient(ambient)
    return o.render(cameras, fov, 1, rgb=True, depth=True, frame=frame, ties=True)["ties"]


def assert_same_tlas(got, want):
    assert np.array_equal(got["keys"], want["keys"])
    assert np.array_equal(got["sorted_ids"], want["sorted_ids"])
    assert np.array_equal(got["roots"], want["roots"])
    assert np.array_equal(got["nodes"][:, [3, 7]], want["nodes"][:, [3, 7]])
    gb, wb = got["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32), want["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32)
    assert np.array_equal(gb, wb)  # float equality: -0 and +0 are the same box
    assert np.array_equal(bits(got["matrices"]), bits(want["matrices"]))


@pytest.mark.parametrize("build", [1, 2])
@pytest.mark.parametrize("case", ["icospheres", "scattered", "coincident", "single_leaf", "bodies", "one_world"])
def test_tree_build_is_the_oracles(torch_cuda, case, build):
    """Both tree builds, the per-world groups (1) and the global build (2), against the oracle."""
    check_tree_build(case, build)


@pytest.mark.parametrize("case", ["large_world", "large_worlds"])
def test_global_build_of_large_worlds_is_the_oracles(torch_cuda, case):
    """Worlds beyond the per-world build's 1024 instances take the global build automatically."""
    check_tree_build(case, 0)


def check_tree_build(case, build):
    if case == "icospheres":
        wl = workloads.icosphere_worlds()
        desc, mats = wl.desc, wl.matrices
    elif case == "scattered":
        desc, mats, _ = scenes.scattered_boxes(300, 40)
    elif case == "coincident":
        desc, mats, _ = scenes.coincident_boxes()
    elif case == "single_leaf":
        desc, mats, _ = scenes.single_leaf_worlds()
    elif case == "one_world":
        desc, mats, _ = scenes.scattered_boxes(1, 1000)
    elif case == "large_world":
        desc, mats, _ = scenes.scattered_boxes(1, 5000)
    elif case == "large_worlds":
        desc, mats, _ = scenes.scattered_boxes(3, 1500)
    else:
        wl = workloads.body_worlds(worlds=256)
        desc, mats = wl.desc, None
    r, o = product(desc), O.Oracle(desc)
    r.set_build(build)
    if mats is not None:
        r.set_instance_transforms(mats)
        o.set_instance_transforms(mats)
    else:
        steps = workloads.random_walk(wl.poses, 2)
        r.bind_bodies(**wl.binding)
        o.bind_bodies(**wl.binding)
        for s in steps:
            r.set_body_poses(s)
            o.set_body_poses(s)
    assert_same_tlas(r.inspect_tlas(), o.tlas())


def test_render_icospheres_is_the_oracles_and_the_references(torch_cuda):
    f = np.load(os.path.join(GOLDEN, "icosphere_16x8_seed0.npz"))
    wl = workloads.icosphere_worlds()
    r, o = product(wl.desc), O.Oracle(wl.desc)
    r.set_instance_transforms(f["matrices"])
    o.set_instance_transforms(f["matrices"])
    r.record_hits(True)
    got = r.render(f["cameras"], float(f["fov"]), 1, **ALL)
    want = o.render(f["cameras"], float(f["fov"]), 1, **ALL, hits=True, ties=True)
    assert_same_images(got, want, ties=want["ties"])
    assert_same_images(got, {k: f[k] for k in ("rgb", "depth", "normals", "object_ids")}, ties=want["ties"])
    assert_same_hits(r.inspect_hits(), want)


def assert_same_hits(h, want):
    ok = (want["ties"] & (O.TIE_AOV_INSTANCE | O.TIE_AOV_TRIANGLE)) == 0 if "ties" in want else slice(None)
    for k in ("hit_instance", "hit_triangle"):
        assert np.array_equal(h[k][ok], want[k][ok]), k
    for k in ("hit_u", "hit_v"):
        assert np.array_equal(bits(h[k][ok]), bits(want[k][ok])), k


def test_render_reference_test_scene(torch_cuda):
    """Spheres, a mirror sphere (reflection bounces), two hard-shadow lights, a checker floor, smooth normals,
    ambient 0.1, 2 samples per pixel, frame 5: against the reference's own images."""
    f = np.load(os.path.join(GOLDEN, "template_6w_spp2_frame5.npz"))
    r = product(scenes.template(worlds=6))
    r.set_instance_transforms(f["matrices"])
    r.ambient = float(f["ambient"])
    got = r.render(f["cameras"], float(f["fov"]), 2, **ALL, frame=5)
    assert_same_images(got, {k: f[k] for k in ("rgb", "depth", "normals", "object_ids")})


def test_body_poses_and_rays_against_the_reference(torch_cuda):
    f = np.load(os.path.join(GOLDEN, "body_16x20_seed0.npz"))
    wl = workloads.body_worlds(worlds=16, seed=0)
    r = product(wl.desc)
    r.bind_bodies(**wl.binding)
    r.set_body_poses(f["poses"])
    assert np.array_equal(bits(r.inspect_tlas()["matrices"].reshape(f["matrices"].shape)), bits(f["matrices"]))
    got = r.render(f["cameras"], float(f["fov"]), 1, rgb=True, depth=True, object_ids=True)
    ties = oracle_ties(wl.desc, f["cameras"], float(f["fov"]), binding=wl.binding, poses=f["poses"])
    assert_same_images(got, {k: f[k] for k in ("rgb", "depth", "object_ids")}, ties=ties)
    hits = r.cast_rays(f["ray_origins"], f["ray_directions"], 20.0)
    assert np.array_equal(hits["object_id"], f["ray_object_id"])
    assert np.array_equal(bits(hits["distance"]), bits(f["ray_distance"]))
    assert np.array_equal(bits(hits["normal"]), bits(f["ray_normal"]))


def test_scattered_worlds_against_the_oracle(torch_cuda):
    desc, mats, cams = scenes.scattered_boxes(300, 40)
    r, o = product(desc), O.Oracle(desc)
    r.set_instance_transforms(mats)
    o.set_instance_transforms(mats)
    assert_same_images(r.render(cams, scenes.FOV, 1, **ALL), o.render(cams, scenes.FOV, 1, **ALL))


def test_known_answers(torch_cuda):
    desc, mats, cams = scenes.one_box_worlds()
    r = product(desc)
    r.set_instance_transforms(mats)
    d = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[:, scenes.H // 2, scenes.W // 2] == pytest.approx([7.0, 2.0], abs=0.02)
    hits = r.cast_rays(np.zeros((2, 1, 3), np.float32), np.tile(np.float32([0, 0, -1]), (2, 1, 1)), 100.0)
    assert hits["distance"][:, 0] == pytest.approx([7.0, 2.0], abs=1e-3)
    assert (hits["object_id"] == ng.OBJECT_INSTANCE).all()
    desc, mats, cams = scenes.single_leaf_worlds()
    r = product(desc)
    r.set_instance_transforms(mats)
    d = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[:, scenes.H // 2, scenes.W // 2] == pytest.approx([3.0, 4.0, 5.0, 6.0], abs=0.02)
    desc, mats, cams = scenes.coincident_boxes()
    r = product(desc)
    r.set_instance_transforms(mats)
    d = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[0, scenes.H // 2, scenes.W // 2] == pytest.approx(4.8, abs=0.02)


def test_worlds_without_instances(torch_cuda):
    desc = scenes.template(worlds=3)
    desc = ng.SceneDesc(desc.width, desc.height, 3, 1, desc.spheres, desc.lights, desc.floor)
    r = product(desc)
    r.set_instance_transforms(np.zeros((0,), np.float32))
    cams = np.stack([scenes.camera()] * 3)
    got = r.render(cams, scenes.FOV, 1, **ALL)
    want = O.Oracle(desc).render(cams, scenes.FOV, 1, **ALL)
    assert_same_images(got, want)


def test_many_worlds_several_cameras(torch_cuda):
    desc = scenes.template(worlds=200, cameras_per_world=2)
    mats = scenes.template_matrices(200)
    cams = np.stack([scenes.camera((0.3 * (v % 2), 0.5, 0)) for v in range(400)])
    r, o = product(desc), O.Oracle(desc)
    r.set_instance_transforms(mats)
    o.set_instance_transforms(mats)
    out = dict(rgb=False, depth=True, object_ids=True)
    assert_same_images(r.render(cams, scenes.FOV, 1, **out), o.render(cams, scenes.FOV, 1, **out))


def test_device_inputs_and_zero_copy(torch_cuda):
    torch = torch_cuda
    wl = workloads.icosphere_worlds()
    d = wl.desc
    host, dev = product(d), product(d)
    host.set_instance_transforms(wl.matrices)
    dev.set_instance_transforms(torch.from_numpy(wl.matrices).cuda())
    want = host.render(wl.cameras, wl.fov, 1, **ALL)
    got = dev.render(torch.from_numpy(wl.cameras).cuda(), wl.fov, 1, **ALL, zero_copy=True)
    assert all(v.is_cuda for v in got.values()) and tuple(got["rgb"].shape) == (16, 64, 64, 3)
    assert_same_images({k: v.cpu().numpy() for k, v in got.items()}, want, rgb_tol=0)
    first = got["depth"]
    kept = first.clone()
    second = dev.render(torch.from_numpy(wl.cameras[::-1].copy()).cuda(), wl.fov, 1, rgb=False, depth=True,
                        zero_copy=True)["depth"]
    assert second.data_ptr() == first.data_ptr() and not torch.equal(first, kept)
    with pytest.raises(ValueError, match="cameras on the GPU need zero_copy=True"):
        dev.render(torch.from_numpy(wl.cameras).cuda(), wl.fov)
    # Matrices given in device memory are the ones inspection reports, on both builds.
    moved = wl.matrices.copy()
    moved[..., 3] += np.float32(0.25)
    for build in (1, 2):
        dev.set_build(build)
        dev.set_instance_transforms(torch.from_numpy(moved).cuda())
        assert np.array_equal(bits(dev.inspect_tlas()["matrices"].reshape(moved.shape)), bits(moved))


def test_body_poses_from_a_gpu_tensor(torch_cuda):
    torch = torch_cuda
    wl = workloads.body_worlds(worlds=64)
    a, b, o = product(wl.desc), product(wl.desc), O.Oracle(wl.desc)
    for x in (a, b, o):
        x.bind_bodies(**wl.binding)
    a.set_body_poses(wl.poses)
    b.set_body_poses(torch.from_numpy(wl.poses).cuda())
    o.set_body_poses(wl.poses)
    assert_same_tlas(b.inspect_tlas(), o.tlas())
    out = dict(rgb=True, depth=True, object_ids=True)
    assert_same_images(b.render(wl.cameras, 1.0, 1, **out), a.render(wl.cameras, 1.0, 1, **out), rgb_tol=0)
    want = o.render(wl.cameras, 1.0, 1, **out, ties=True)
    assert_same_images(b.render(wl.cameras, 1.0, 1, **out), want, ties=want["ties"])


def test_rejected_input_changes_nothing(torch_cuda):
    desc = scenes.template(worlds=2)
    mats = scenes.template_matrices(2)
    r = product(desc)
    r.set_instance_transforms(mats)
    cams = np.stack([scenes.camera((0, 0, 0))] * 2)
    before = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"].copy()
    singular = mats.copy()
    singular[1, 1] = 0
    with pytest.raises(ValueError, match="world 1 instance 1 transform is singular"):
        r.set_instance_transforms(singular)
    bad = mats.copy()
    bad[0, 2, 1, 3] = np.nan
    with pytest.raises(ValueError, match="world 0 instance 2 transform has a NaN or infinite value"):
        r.set_instance_transforms(bad)
    with pytest.raises(ValueError, match="matrices has 12 values, but 72 are needed"):
        r.set_instance_transforms(np.zeros((1, 3, 4), np.float32))
    with pytest.raises(ValueError, match="render needs at least one output"):
        r.render(cams, scenes.FOV, rgb=False)
    with pytest.raises(ValueError, match="samples_per_pixel must be 1 or more, got 0"):
        r.render(cams, scenes.FOV, 0)
    for fov in (0.0, 4.0, float("nan")):
        with pytest.raises(ValueError, match="fov must be between 0 and pi radians"):
            r.render(cams, fov)
    with pytest.raises(ValueError, match="frame must be 0 or more, got -1"):
        r.render(cams, scenes.FOV, frame=-1)
    nan_cam = cams.copy()
    nan_cam[0, 0, 3] = np.nan
    with pytest.raises(ValueError, match="a camera has a NaN or infinite value"):
        r.render(nan_cam, scenes.FOV)
    with pytest.raises(ValueError, match="2 cameras of 3 x 4"):
        r.render(cams[:1], scenes.FOV)
    with pytest.raises(ValueError, match="set_body_poses needs bind_bodies to be called first"):
        r.set_body_poses(np.zeros((2, 2, 7), np.float32))
    with pytest.raises(ValueError, match="instance 2 is on body 5, but there are 1 bodies per world"):
        r.bind_bodies([0, 0, 5], np.tile(np.float32([0, 0, 0, 0, 0, 0, 1]), (3, 1)), np.ones((3, 3)), 1)
    with pytest.raises(ValueError, match="origins must hold 3 floats for each ray"):
        r.cast_rays(np.zeros((1, 3), np.float32), np.zeros((1, 3), np.float32))
    with pytest.raises(ValueError, match="max_distance must be positive"):
        r.cast_rays(np.zeros((2, 1, 3), np.float32), np.ones((2, 1, 3), np.float32), 0.0)
    with pytest.raises(ValueError, match="ambient must be 0 or more"):
        r.ambient = -1.0
    after = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert np.array_equal(bits(after), bits(before))


def test_a_thousand_worlds_stay_in_gpu_memory(torch_cuda):
    torch = torch_cuda
    desc = scenes.template(worlds=1000)
    r = product(desc)
    r.set_instance_transforms(torch.from_numpy(scenes.template_matrices(1000)).cuda())
    cams = torch.from_numpy(np.stack([scenes.camera()] * 1000)).cuda()
    depth = r.render(cams, scenes.FOV, 1, rgb=False, depth=True, zero_copy=True)["depth"]
    assert tuple(depth.shape) == (1000, scenes.H, scenes.W) and depth.is_cuda
    assert float(torch.isfinite(depth).float().mean()) > 0.1
    assert r.last_kernel_ms > 0


@pytest.mark.parametrize("kernel", [1, 2, 3])
def test_every_render_kernel_is_the_oracles(torch_cuda, kernel):
    """The per-pixel, persistent and tile kernels, forced in turn, on odd image sizes (partial tiles), two
    cameras per world, spheres and a checker floor, with hit records."""
    wl = workloads.icosphere_worlds(worlds=5, width=37, height=29, seed=11)
    d = wl.desc
    spheres = [ng.Sphere((0.5, -1.0, -7.0), 0.7), ng.Sphere((-1.5, 0.0, -8.0), 0.5)]
    floor = ng.Plane(y=-2.0, half_extent_x=12.0, z_min=-30.0, z_max=-2.0, checker_scale=1.0)
    desc = ng.SceneDesc(d.width, d.height, 5, 2, spheres, d.lights, floor, d.meshes, d.instances)
    cams = np.repeat(wl.cameras, 2, axis=0)
    cams[1::2, :, 3] += np.float32([0.3, 0.0, 0.0])
    r, o = product(desc), O.Oracle(desc)
    if kernel == 3:
        r.set_tuning(kernel=3, threads_per_block=128, registers=64)
    else:
        r.set_tuning(kernel=kernel, threads_per_block=128, refill_lanes=8, registers=48)
    r.set_instance_transforms(wl.matrices)
    o.set_instance_transforms(wl.matrices)
    r.ambient = 0.05
    o.set_ambient(0.05)
    r.record_hits(True)
    got = r.render(cams, 1.0, 1, **ALL, frame=3)
    want = o.render(cams, 1.0, 1, **ALL, frame=3, hits=True, ties=kernel == 3)
    assert_same_images(got, want, ties=want.get("ties"))
    assert_same_hits(r.inspect_hits(), want)


@pytest.mark.parametrize("kernel", [2, 3])
@pytest.mark.parametrize("outputs", [dict(rgb=True), dict(rgb=False, depth=True), dict(rgb=False, object_ids=True)])
def test_one_kind_of_output(torch_cuda, outputs, kernel):
    wl = workloads.body_worlds(worlds=64, seed=2)
    r, o = product(wl.desc), O.Oracle(wl.desc)
    for x in (r, o):
        x.bind_bodies(**wl.binding)
        x.set_body_poses(wl.poses)
    r.set_tuning(kernel=kernel, registers=72 if kernel == 2 else 80)
    want = o.render(wl.cameras, 1.0, 1, **outputs)
    ties = oracle_ties(wl.desc, wl.cameras, binding=wl.binding, poses=wl.poses) if kernel == 3 else None
    assert_same_images(r.render(wl.cameras, 1.0, 1, **outputs), want, ties=ties)


def test_persistent_kernel_tunings_agree(torch_cuda):
    wl = workloads.body_worlds(worlds=128, seed=5)
    r = product(wl.desc)
    r.bind_bodies(**wl.binding)
    r.set_body_poses(wl.poses)
    out = dict(rgb=True, depth=True, object_ids=True)
    r.set_tuning(kernel=1)
    want = r.render(wl.cameras, 1.0, 1, **out)
    for threads, refill, regs, batch in ((256, 16, 64, 1), (128, 4, 72, 32), (64, 32, 64, 8), (128, 1, 48, 16),
                                         (256, 24, 48, 24)):
        r.set_tuning(kernel=2, threads_per_block=threads, refill_lanes=refill, registers=regs, leaf_batch=batch)
        assert_same_images(r.render(wl.cameras, 1.0, 1, **out), want, rgb_tol=0)


def test_tile_kernel_tunings_agree(torch_cuda):
    """Every tile-kernel shape renders the same images bit for bit, and the per-pixel kernel's apart from
    near-ties."""
    wl = workloads.body_worlds(worlds=128, seed=5)
    r = product(wl.desc)
    r.bind_bodies(**wl.binding)
    r.set_body_poses(wl.poses)
    out = dict(rgb=True, depth=True, object_ids=True)
    r.set_tuning(kernel=1)
    ref = r.render(wl.cameras, 1.0, 1, **out)
    ties = oracle_ties(wl.desc, wl.cameras, binding=wl.binding, poses=wl.poses)
    first = None
    for threads, regs in ((128, 48), (128, 56), (128, 64), (128, 80), (256, 64)):
        r.set_tuning(kernel=3, threads_per_block=threads, registers=regs)
        got = r.render(wl.cameras, 1.0, 1, **out)
        assert_same_images(got, ref, ties=ties)
        if first is None:
            first = got
        else:
            assert_same_images(got, first, rgb_tol=0)
    for fetch in (1, 2, 3, 8):
        for paired in (True, False):
            r.set_tuning(kernel=3, threads_per_block=128, registers=56)
            r.set_tile_shape(fetch, paired)
            assert_same_images(r.render(wl.cameras, 1.0, 1, **out), first, rgb_tol=0)


def test_tile_shapes_agree_on_uneven_worlds(torch_cuda):
    """Tiles per fetch and paired or one-kind camera tiles: the same images bit for bit on worlds of uneven sizes."""
    worlds, meshes, floor, lights, mats, cams = uneven_scene(seed=6)
    u = ng.UnevenBatchRenderer(worlds, lights=lights, floor=floor, meshes=meshes, device="cuda:0")
    u.set_instance_transforms(mats)
    first = u.render(cams, 1.0, 1, **ALL, frame=1)
    for fetch in (1, 2, 4):
        for paired in (True, False):
            u.set_tile_shape(fetch, paired)
            got = u.render(cams, 1.0, 1, **ALL, frame=1)
            for k in first:
                assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8),
                                      np.ascontiguousarray(first[k]).view(np.uint8)), (k, fetch, paired)


def test_tile_kernel_on_worlds_of_one_to_256_instances(torch_cuda):
    """The tile kernel's cases: worlds of one instance (the root is the only leaf), exactly 32 (one per lane),
    33 (a second chunk of candidates) and 256 (the largest it takes, eight chunks)."""
    for per_world in (1, 32, 33, 256):
        wl = workloads.icosphere_worlds(worlds=6, per_world=per_world, width=40, height=24, seed=13)
        r, o = product(wl.desc), O.Oracle(wl.desc)
        r.set_tuning(kernel=3, threads_per_block=256, registers=64)
        r.set_instance_transforms(wl.matrices)
        o.set_instance_transforms(wl.matrices)
        want = o.render(wl.cameras, 1.0, 1, **ALL, ties=True)
        assert_same_images(r.render(wl.cameras, 1.0, 1, **ALL), want, ties=want["ties"])


def test_large_world_renders_and_casts_rays(torch_cuda):
    """One world of 3000 instances (global build, the persistent kernel's world-tree walk): images and a LiDAR
    sweep against the oracle."""
    desc, mats, cams = scenes.scattered_boxes(1, 3000)
    r, o = product(desc), O.Oracle(desc)
    r.set_instance_transforms(mats)
    o.set_instance_transforms(mats)
    want = o.render(cams, scenes.FOV, 1, **ALL, ties=True)
    assert_same_images(r.render(cams, scenes.FOV, 1, **ALL), want, ties=want["ties"])
    el = np.radians(np.linspace(-15.0, 15.0, 16))
    az = np.radians(np.linspace(0.0, 360.0, 128, endpoint=False))
    e, a = np.meshgrid(el, az, indexing="ij")
    dirs = np.stack([np.cos(e) * np.sin(a), np.sin(e), -np.cos(e) * np.cos(a)], -1).reshape(1, -1, 3).astype(np.float32)
    origins = np.tile(np.float32([0.0, 0.0, -40.0]), (1, dirs.shape[1], 1))
    exp = o.cast_rays(origins, dirs, 100.0)
    for kernel in (0, 2, 1):  # automatic (warp packets in a world this large), persistent, per thread
        r.set_ray_kernel(kernel)
        got = r.cast_rays(origins, dirs, 100.0)
        assert (got["object_id"] >= 34).mean() > 0.2
        assert np.array_equal(got["object_id"], exp["object_id"])
        assert np.array_equal(bits(got["distance"]), bits(exp["distance"]))
        assert np.array_equal(bits(got["normal"]), bits(exp["normal"]))


def uneven_scene(seed=4):
    """Seven worlds of 0 to 200 instances of three meshes at five image sizes, with their cameras and matrices."""
    rng = np.random.default_rng(seed)
    meshes = [ng.make_box((0.4, 0.4, 0.4)), ng.make_icosphere(0.5, 2), ng.cylinder(1.0, 1.0, 32)]
    counts = [1, 5, 33, 0, 12, 200, 3]
    sizes = [(32, 32), (64, 64), (48, 40), (64, 64), (128, 128), (64, 48), (40, 24)]
    worlds, mats, cams = [], [], []
    for w, (count, (width, height)) in enumerate(zip(counts, sizes)):
        insts = [ng.Instance(int(rng.integers(0, 3)), material=ng.Material(diffuse_color=tuple(rng.uniform(0.2, 0.9, 3))))
                 for _ in range(count)]
        worlds.append((width, height, insts))
        for i in range(count):
            q = rng.normal(size=4)
            mats.append(ng.make_transform(rng.uniform(-2, 2, 3) + (0, 0, -6), q / np.linalg.norm(q),
                                          float(rng.uniform(0.3, 0.8))).matrix)
        eye = np.array([0.0, 1.0, 0.0]) + rng.uniform(-0.3, 0.3, 3)
        cams.append(workloads.camera_matrix(eye, (0.0, 0.0, -6.0), width, height, 1.0))
    floor = ng.Plane(y=-2.5, half_extent_x=12.0, z_min=-30.0, z_max=-2.0, checker_scale=1.0)
    lights = [ng.Light((-10.0, 20.0, 10.0), 1.6, 1.0)]
    return worlds, meshes, floor, lights, np.stack(mats).astype(np.float32), np.stack(cams).astype(np.float32)


def test_uneven_worlds_are_each_worlds_own_render(torch_cuda):
    """One uneven renderer against, world by world, a plain renderer of that world alone (bit for bit: the
    same kernels see the same world) and the oracle (apart from near-ties)."""
    worlds, meshes, floor, lights, mats, cams = uneven_scene()
    u = ng.UnevenBatchRenderer(worlds, lights=lights, floor=floor, meshes=meshes, device="cuda:0")
    u.set_instance_transforms(mats)
    got = u.render(cams, 1.0, 1, **ALL, frame=2)
    assert got["depth"].shape == (u.pixel_count,)
    first = u.instance_first
    for w, (width, height, insts) in enumerate(worlds):
        desc = ng.SceneDesc(width, height, 1, 1, [], lights, floor, meshes, insts)
        m = mats[first[w]:first[w + 1]].reshape(1, len(insts), 3, 4)
        mine = {k: u.image(v, w)[None] for k, v in got.items()}
        plain = product(desc)
        if insts:
            plain.set_instance_transforms(m)
        assert_same_images(mine, plain.render(cams[w:w + 1], 1.0, 1, **ALL, frame=2), rgb_tol=0)
        o = O.Oracle(desc)
        if insts:
            o.set_instance_transforms(m)
        want = o.render(cams[w:w + 1], 1.0, 1, **ALL, frame=2, ties=True)
        assert_same_images(mine, want, ties=want["ties"])


def test_uneven_step_captured_in_a_cuda_graph_is_the_eager_step(torch_cuda):
    """One uneven step (every world's tree build and the render's kernels) captured into a CUDA graph, replayed
    after the matrices changed in place: RGB, depth and IDs bit for bit those of the same step run eagerly, and
    those of the oracle (apart from near ties)."""
    torch = torch_cuda
    worlds, meshes, floor, lights, mats, cams = uneven_scene(seed=8)
    u = ng.UnevenBatchRenderer(worlds, lights=lights, floor=floor, meshes=meshes, device="cuda:0")
    moved = mats.copy()
    rng = np.random.default_rng(2)
    moved[:, :, 3] += rng.normal(0.0, 0.05, size=moved[:, :, 3].shape).astype(np.float32)
    static = torch.from_numpy(mats).cuda()
    cams_dev = torch.from_numpy(cams).cuda()
    kw = dict(rgb=True, depth=True, object_ids=True, zero_copy=True, frame=4)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            u.set_instance_transforms(static)
            u.render(cams_dev, 1.0, 1, **kw)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        u.set_instance_transforms(static)
        out = u.render(cams_dev, 1.0, 1, **kw)
    static.copy_(torch.from_numpy(moved))
    graph.replay()
    torch.cuda.synchronize()
    replayed = {k: v.cpu().numpy() for k, v in out.items()}
    u.set_instance_transforms(moved)
    eager = u.render(cams, 1.0, 1, rgb=True, depth=True, object_ids=True, frame=4)
    for k in ("rgb", "depth", "object_ids"):
        a, b = np.ascontiguousarray(replayed[k]), np.ascontiguousarray(eager[k])
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    first = u.instance_first
    for w, (width, height, insts) in enumerate(worlds):
        desc = ng.SceneDesc(width, height, 1, 1, [], lights, floor, meshes, insts)
        o = O.Oracle(desc)
        if insts:
            o.set_instance_transforms(moved[first[w]:first[w + 1]].reshape(1, len(insts), 3, 4))
        want = o.render(cams[w:w + 1], 1.0, 1, rgb=True, depth=True, object_ids=True, frame=4, ties=True)
        assert_same_images({k: u.image(v, w)[None] for k, v in replayed.items()}, want, ties=want["ties"])


def test_ray_queries_on_both_kernels(torch_cuda):
    """Ray queries through the persistent kernel's walk (the default here), the per-thread kernel and warp
    packets: the same distances, normals and IDs, with rays of zero length, rays stopped by max_distance and rays
    in worlds of their own (500 rays a world: a partial packet at each world's end)."""
    wl = workloads.body_worlds(worlds=8, seed=6)
    r, o = product(wl.desc), O.Oracle(wl.desc)
    for x in (r, o):
        x.bind_bodies(**wl.binding)
        x.set_body_poses(wl.poses)
    rng = np.random.default_rng(3)
    origins = rng.uniform(-3.0, 3.0, size=(8, 500, 3)).astype(np.float32)
    dirs = rng.normal(size=(8, 500, 3)).astype(np.float32)
    dirs[:, ::50] = 0.0  # no direction: a miss
    want = o.cast_rays(origins, dirs, 4.0)
    got = r.cast_rays(origins, dirs, 4.0)
    r.set_ray_kernel(3)
    packets = r.cast_rays(origins, dirs, 4.0)
    r.set_ray_kernel(0)
    r.set_tuning(kernel=1)
    per_thread = r.cast_rays(origins, dirs, 4.0)
    assert (want["object_id"] > 0).mean() > 0.2 and np.isinf(want["distance"]).mean() > 0.1
    for k in ("object_id", "distance", "normal"):
        for each in (got, per_thread, packets):
            assert np.array_equal(np.asarray(each[k]).view(np.uint32), np.asarray(want[k]).view(np.uint32)), k


def l_prism(depth=0.6):
    """A concave mesh: an L-shaped outline (2 x 2 with a 1 x 1 notch) extruded along z, 20 triangles."""
    outline = np.float32([[0, 0], [2, 0], [2, 1], [1, 1], [1, 2], [0, 2]]) - np.float32(0.8)
    verts = np.concatenate([np.c_[outline, np.full(6, -depth)], np.c_[outline, np.full(6, depth)]]).astype(np.float32)
    tris = [(0, i, i + 1) for i in range(1, 5)] + [(6, 6 + i + 1, 6 + i) for i in range(1, 5)]
    for i in range(6):
        j = (i + 1) % 6
        tris += [(i, j, 6 + j), (i, 6 + j, 6 + i)]
    return ng.Mesh(verts, np.uint32(tris))


def open_bowl(radius=0.7, rings=6, segments=16):
    """An open mesh: the lower half of a sphere, without a lid, so it is seen from inside and outside."""
    verts = [(0.0, -radius, 0.0)]
    for k in range(1, rings + 1):
        a = 0.5 * np.pi * k / rings
        for j in range(segments):
            b = 2 * np.pi * j / segments
            verts.append((radius * np.sin(a) * np.cos(b), -radius * np.cos(a), radius * np.sin(a) * np.sin(b)))
    tris = [(0, 1 + j, 1 + (j + 1) % segments) for j in range(segments)]
    for k in range(1, rings):
        a0, a1 = 1 + (k - 1) * segments, 1 + k * segments
        for j in range(segments):
            jn = (j + 1) % segments
            tris += [(a0 + j, a1 + j, a1 + jn), (a0 + j, a1 + jn, a0 + jn)]
    return ng.Mesh(np.float32(verts), np.uint32(tris))


@pytest.mark.parametrize("light_y", [20.0, -1.0])
def test_shadows_of_convex_concave_and_open_meshes(torch_cuda, light_y):
    """Shadow rays leaving convex meshes (box, smooth icosphere), a concave one (an L prism, which shadows
    itself) and an open bowl, under shears and uneven scales, with the light high (most surfaces lit) and low
    (many lit from behind, the shadow ray starting inside its own mesh): the oracle's images on every kernel."""
    rng = np.random.default_rng(21)
    meshes = [ng.make_box((0.5, 0.3, 0.4)), ng.make_icosphere(0.6, 2), l_prism(), open_bowl()]
    per_world, worlds = 12, 6
    instances = [ng.Instance(i % 4, material=ng.Material(diffuse_color=workloads.PALETTE[i % 8])) for i in range(per_world)]
    floor = ng.Plane(y=-2.0, half_extent_x=10.0, z_min=-20.0, z_max=2.0, checker_scale=1.0)
    lights = [ng.Light((3.0, light_y, -2.0), 1.5, 0.0)]
    desc = ng.SceneDesc(48, 40, worlds, 1, [], lights, floor, meshes, instances)
    mats = np.empty((worlds, per_world, 3, 4), np.float32)
    for w in range(worlds):
        for i in range(per_world):
            m = ng.make_transform(rng.uniform([-2.5, -1.5, -8.0], [2.5, 1.5, -4.0]), rng.normal(size=4),
                                  1.0).matrix
            shear = np.eye(3, dtype=np.float32) + np.float32(rng.uniform(-0.4, 0.4, (3, 3)) * (1 - np.eye(3)))
            m[:, :3] = m[:, :3] @ (shear * np.float32(rng.uniform(0.5, 1.5, 3)))
            mats[w, i] = m
    cams = np.stack([workloads.camera_matrix(rng.uniform(-0.5, 0.5, 3) + (0.0, 1.0, 0.0), (0.0, 0.0, -6.0), 48, 40,
                                             1.0) for _ in range(worlds)]).astype(np.float32)
    o = O.Oracle(desc)
    o.set_instance_transforms(mats)
    want = o.render(cams, 1.0, 1, **ALL, ties=True)
    ids = want["object_ids"]
    assert len(np.unique(ids[ids > 0])) >= 10  # most instances and the floor are in view
    for kernel in (1, 2, 3):
        r = product(desc)
        r.set_tuning(kernel=kernel, threads_per_block=128, refill_lanes=8, registers=64)
        r.set_instance_transforms(mats)
        assert_same_images(r.render(cams, 1.0, 1, **ALL), want, ties=want["ties"] if kernel == 3 else None)


@pytest.mark.parametrize("tuning", [(128, 56), (256, 64)])
def test_tile_kernel_walks_large_worlds_as_packets(torch_cuda, tuning):
    """Worlds above 256 instances on the tile kernels: the world tree walked by the warp as a packet for the
    camera rays and the shadow rays, against the oracle (one world of 3000 boxes, global build; three worlds of
    400 icospheres, per-world build)."""
    desc, mats, cams = scenes.scattered_boxes(1, 3000)
    cases = [(desc, mats, cams, scenes.FOV)]
    wl = workloads.icosphere_worlds(worlds=3, per_world=400, width=48, height=40, seed=17)
    cases.append((wl.desc, wl.matrices, wl.cameras, 1.0))
    for d, m, c, fov in cases:
        r, o = product(d), O.Oracle(d)
        r.set_tuning(kernel=3, threads_per_block=tuning[0], registers=tuning[1])
        r.set_instance_transforms(m)
        o.set_instance_transforms(m)
        want = o.render(c, fov, 1, **ALL, ties=True)
        got = r.render(c, fov, 1, **ALL)
        assert (got["object_ids"] >= 34).mean() > 0.1
        assert_same_images(got, want, ties=want["ties"])


def test_packet_tiles_with_partial_tiles_two_cameras_spheres_and_floor(torch_cuda):
    """The large-world tile path with everything around it: 300 instances per world (packet walk), two cameras
    per world, 37x29 images (partial tiles), spheres and a checker floor, shadow rays as persistent-kernel
    pixel jobs: against the oracle."""
    wl = workloads.icosphere_worlds(worlds=3, per_world=300, width=37, height=29, seed=23)
    d = wl.desc
    spheres = [ng.Sphere((0.5, -1.0, -7.0), 0.7), ng.Sphere((-1.5, 0.0, -8.0), 0.5)]
    floor = ng.Plane(y=-2.0, half_extent_x=12.0, z_min=-30.0, z_max=-2.0, checker_scale=1.0)
    desc = ng.SceneDesc(d.width, d.height, 3, 2, spheres, d.lights, floor, d.meshes, d.instances)
    cams = np.repeat(wl.cameras, 2, axis=0)
    cams[1::2, :, 3] += np.float32([0.4, 0.1, 0.0])
    r, o = product(desc), O.Oracle(desc)
    r.set_instance_transforms(wl.matrices)
    o.set_instance_transforms(wl.matrices)
    r.ambient = 0.05
    o.set_ambient(0.05)
    want = o.render(cams, 1.0, 1, **ALL, frame=2, ties=True)
    got = r.render(cams, 1.0, 1, **ALL, frame=2)
    assert (got["object_ids"] >= 34).mean() > 0.1 and (got["object_ids"] == 33).mean() > 0.01
    assert_same_images(got, want, ties=want["ties"])


@pytest.mark.parametrize("per_world", [8, 40, 300])
def test_paired_camera_rays_equal_one_kind_at_a_time(torch_cuda, per_world):
    """A render asking for the picture and the centre-ray outputs traces a pixel's two rays on adjacent lanes of a
    4x4 tile; asking for one kind only traces it over 8x4 tiles. Every output is the same bit for bit either
    way (candidate lists of 32 and 256, the packet walk; 37x29 images, partial tiles, two cameras per world)."""
    wl = workloads.icosphere_worlds(worlds=3, per_world=per_world, width=37, height=29, seed=31)
    d = wl.desc
    desc = ng.SceneDesc(d.width, d.height, 3, 2, d.spheres, d.lights, d.floor, d.meshes, d.instances)
    cams = np.repeat(wl.cameras, 2, axis=0)
    cams[1::2, :, 3] += np.float32([0.3, 0.2, 0.1])
    r = product(desc)
    r.set_instance_transforms(wl.matrices)
    both = r.render(cams, 1.0, 1, **ALL, frame=5)
    rgb = r.render(cams, 1.0, 1, rgb=True, frame=5)
    aov = r.render(cams, 1.0, 1, rgb=False, depth=True, normals=True, object_ids=True, frame=5)
    assert (both["object_ids"] >= 34).mean() > 0.1
    assert np.array_equal(both["rgb"], rgb["rgb"])
    for k in ("depth", "normals", "object_ids"):
        assert np.array_equal(both[k].view(np.uint32), aov[k].view(np.uint32)), k


def test_paired_camera_rays_on_uneven_worlds_equal_one_kind_at_a_time(torch_cuda):
    wl = workloads.icosphere_worlds(worlds=3, per_world=12, width=37, height=29, seed=37)
    d = wl.desc
    worlds = [(37, 29, d.instances[:12]), (16, 16, d.instances[:5]), (21, 9, d.instances[:9])]
    u = ng.UnevenBatchRenderer(worlds, lights=d.lights, floor=d.floor, meshes=d.meshes, device="cuda:0")
    m = np.concatenate([wl.matrices[0, :12], wl.matrices[1, :5], wl.matrices[2, :9]]).astype(np.float32)
    u.set_instance_transforms(m)
    both = u.render(wl.cameras, 1.0, **ALL)
    rgb = u.render(wl.cameras, 1.0, rgb=True)
    aov = u.render(wl.cameras, 1.0, rgb=False, depth=True, normals=True, object_ids=True)
    assert (both["object_ids"] >= 34).mean() > 0.05
    assert np.array_equal(both["rgb"], rgb["rgb"])
    for k in ("depth", "normals", "object_ids"):
        assert np.array_equal(both[k].view(np.uint32), aov[k].view(np.uint32)), k
