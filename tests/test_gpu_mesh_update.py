"""Meshes whose vertices move: the device rebuild of a mesh's tree against the host build of the same mesh
(ng.build_meshes, itself checked against the reference's build_meshes), node for node and bit for bit, and
the images of the updated scene against the oracle's images of a scene made with the moved vertices."""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
from neraulgraphics_b200 import scene as S
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu
ALL = dict(rgb=True, depth=True, normals=True, object_ids=True)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def moved(mesh, seed, scale=0.05):
    """The mesh's vertices pushed about: a twist about y, a stretch and per-vertex noise."""
    rng = np.random.default_rng(seed)
    v = mesh.vertices.astype(np.float64)
    a = 0.6 * v[:, 1]
    x = v[:, 0] * np.cos(a) - v[:, 2] * np.sin(a)
    z = v[:, 0] * np.sin(a) + v[:, 2] * np.cos(a)
    out = np.stack([1.3 * x, v[:, 1], z], 1) + rng.normal(scale=scale, size=v.shape)
    return out.astype(np.float32)


def signed_zeros():
    v = np.float32([[0, 0, 0], [-0.0, 1, 0], [0, -0.0, 1], [1, 1, -0.0], [-0.0, -0.0, -0.0]])
    return S.Mesh(v, np.uint32([[0, 1, 2], [1, 3, 4], [4, 2, 0], [3, 2, 1]]))


def meshes():
    rng = np.random.default_rng(5)
    soup = S.Mesh(rng.normal(size=(300, 3)).astype(np.float32), np.arange(300, dtype=np.uint32).reshape(100, 3))
    same = S.Mesh(np.tile(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), (10, 1)), np.arange(30, dtype=np.uint32).reshape(10, 3))
    one = S.Mesh(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), np.uint32([[0, 1, 2]]))
    return [S.make_icosphere(0.5, 3), S.make_box((0.4, 0.3, 0.5)), S.cylinder(1.0, 1.0, 64), soup, same, one,
            signed_zeros()]


def assert_same_tree(got, want):
    assert np.array_equal(got["nodes"], want["nodes"])
    assert np.array_equal(bits(got["triangles"]), bits(want["triangles"]))
    assert np.array_equal(got["triangle_index"], want["triangle_index"])
    assert np.array_equal(bits(got["bounds"][0]), bits(want["bounds"][0]))


def renderer(ms, worlds=2):
    insts = [S.Instance(i, S.make_transform((1.2 * i - 3.0, 0.0, -6.0), (0, 0, 0, 1), 0.8)) for i in range(len(ms))]
    floor = S.Plane(y=-2.0, half_extent_x=12.0, z_min=-30.0, z_max=-2.0, checker_scale=1.0)
    desc = S.SceneDesc(64, 48, worlds, 1, [], [workloads.LIGHT], floor, ms, insts)
    r = ng.BatchRenderer(64, 48, worlds, 1, [], [workloads.LIGHT], floor, ms, insts, device="cuda:0")
    return r, desc, insts, floor


def test_rebuilt_trees_are_the_host_builds(torch_cuda):
    """Every mesh moved and rebuilt on the device (host and CUDA vertex arrays), then moved back: each time
    the tree ng.build_meshes makes of those vertices, including a one-triangle tree, coincident triangles and
    -0 / +0 coordinates."""
    torch = torch_cuda
    ms = meshes()
    r, _, _, _ = renderer(ms)
    for m, mesh in enumerate(ms):
        assert_same_tree(r.inspect_mesh(m), ng.build_meshes([mesh]))
    for m, mesh in enumerate(ms):
        for seed, device in ((1, False), (2, True)):
            v = moved(mesh, seed + m)
            r.update_mesh(m, torch.from_numpy(v).cuda() if device else v)
            assert_same_tree(r.inspect_mesh(m), ng.build_meshes([S.Mesh(v, mesh.triangles)]))
        r.update_mesh(m, mesh.vertices)
        assert_same_tree(r.inspect_mesh(m), ng.build_meshes([mesh]))


def test_a_large_mesh_rebuilt(torch_cuda):
    """20,480 triangles (icosphere subdivision 5): a deep tree, many levels, large partitions."""
    mesh = S.make_icosphere(0.5, 5)
    r, _, _, _ = renderer([mesh], worlds=1)
    v = moved(mesh, 9, scale=0.01)
    r.update_mesh(0, v)
    assert_same_tree(r.inspect_mesh(0), ng.build_meshes([S.Mesh(v, mesh.triangles)]))


def test_images_after_an_update_are_the_oracles(torch_cuda):
    """The updated renderer's trees and images against the oracle's of a scene made with the moved vertices:
    instance trees rebuilt around the meshes' new boxes, hits on the moved triangles, on every kernel."""
    ms = [S.make_icosphere(0.5, 2), S.make_box((0.4, 0.3, 0.5)), S.cylinder(1.0, 1.0, 32)]
    new = [S.Mesh(moved(m, 3 + i, scale=0.03) * np.float32(1.4), m.triangles) for i, m in enumerate(ms)]
    r, desc, insts, floor = renderer(ms, worlds=3)
    rng = np.random.default_rng(2)
    mats = np.stack([[S.make_transform(rng.uniform([-2.5, -1.0, -7.0], [2.5, 1.0, -5.0]), rng.normal(size=4),
                                       1.0).matrix for _ in ms] for _ in range(3)]).astype(np.float32)
    cams = np.stack([workloads.camera_matrix((0.3 * w, 0.8, 0.0), (0.0, 0.0, -6.0), 64, 48, 1.0)
                     for w in range(3)]).astype(np.float32)
    r.set_instance_transforms(mats)
    for i, m in enumerate(new):
        r.update_mesh(i, m.vertices)
    o = O.Oracle(S.SceneDesc(64, 48, 3, 1, [], [workloads.LIGHT], floor, new, insts))
    o.set_instance_transforms(mats)
    got_t, want_t = r.inspect_tlas(), o.tlas()
    for k in ("keys", "sorted_ids", "roots"):
        assert np.array_equal(got_t[k], want_t[k]), k
    assert np.array_equal(got_t["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32),
                          want_t["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32))
    for kernel in (1, 2, 3):
        r.set_tuning(kernel=kernel, threads_per_block=128, refill_lanes=8, registers=64)
        want = o.render(cams, 1.0, 1, **ALL, ties=kernel == 3)
        got = r.render(cams, 1.0, 1, **ALL)
        ok = np.ones(got["depth"].shape, bool) if kernel != 3 else (want["ties"] & O.TIE_AOV_INSTANCE) == 0
        assert np.array_equal(got["object_ids"][ok], want["object_ids"][ok])
        assert np.array_equal(bits(got["depth"][ok]), bits(want["depth"][ok]))
        assert np.array_equal(bits(got["normals"][ok]), bits(want["normals"][ok]))
        rgb_ok = ok if kernel != 3 else (want["ties"] & O.TIE_RGB_INSTANCE) == 0
        assert np.abs(got["rgb"].astype(int) - want["rgb"].astype(int)).max(-1)[rgb_ok].max(initial=0) <= 1


def test_vertex_normals_follow_the_update(torch_cuda):
    """A smooth-shaded mesh: new vertex normals given with the vertices are the ones the normals image shows."""
    base = S.make_icosphere(0.5, 2)
    normals = base.vertices / np.linalg.norm(base.vertices, axis=1, keepdims=True)
    mesh = S.Mesh(base.vertices, base.triangles, normals)
    r, _, insts, floor = renderer([mesh, S.make_box((0.3, 0.3, 0.3))], worlds=1)
    v = moved(base, 4, scale=0.0) * np.float32([1.5, 0.7, 1.0])
    n = (v / np.float32([1.5 ** 2, 0.7 ** 2, 1.0])).astype(np.float32)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    r.update_mesh(0, v, n)
    o = O.Oracle(S.SceneDesc(64, 48, 1, 1, [], [workloads.LIGHT], floor, [S.Mesh(v, base.triangles, n),
                                                                          S.make_box((0.3, 0.3, 0.3))], insts))
    o.set_instance_transforms(np.stack([[i.transform.matrix for i in insts]]).astype(np.float32))
    cams = workloads.camera_matrix((-3.0, 0.6, -4.0), (-3.0, 0.0, -6.0), 64, 48, 1.0)[None].astype(np.float32)
    r.set_tuning(kernel=1)
    got, want = r.render(cams, 1.0, 1, **ALL), o.render(cams, 1.0, 1, **ALL)
    assert (got["object_ids"] == 34).mean() > 0.05
    assert np.array_equal(bits(got["normals"]), bits(want["normals"]))
    assert np.array_equal(bits(got["depth"]), bits(want["depth"]))


def test_update_arguments_are_checked(torch_cuda):
    ms = [S.make_box((0.4, 0.4, 0.4)), S.make_icosphere(0.5, 1)]
    r, _, _, _ = renderer(ms)
    before = r.inspect_mesh(1)
    bad = ms[1].vertices.copy()
    bad[7, 2] = np.inf
    with pytest.raises(ValueError, match="mesh 1 vertex 7 has a NaN or infinite value"):
        r.update_mesh(1, bad)
    assert_same_tree(r.inspect_mesh(1), before)
    with pytest.raises(ValueError, match="mesh 1 has 42 vertices"):
        r.update_mesh(1, bad[:40])
    with pytest.raises(ValueError, match="mesh 2 does not exist"):
        r.update_mesh(2, bad)
    with pytest.raises(ValueError, match="made without vertex normals"):
        r.update_mesh(0, ms[0].vertices, ms[0].vertices)


def test_uneven_worlds_follow_a_mesh_update(torch_cuda):
    """Worlds of uneven sizes: a moved mesh in every world that uses it (slot tables per instance), against a
    plain renderer of each world made with the moved mesh, bit for bit."""
    import test_gpu_parity as P
    worlds, meshes, floor, lights, mats, cams = P.uneven_scene()
    u = ng.UnevenBatchRenderer(worlds, lights=lights, floor=floor, meshes=meshes, device="cuda:0")
    u.set_instance_transforms(mats)
    new = list(meshes)
    new[1] = S.Mesh(moved(meshes[1], 12, scale=0.02) * np.float32(1.3), meshes[1].triangles)
    u.update_mesh(1, new[1].vertices)
    got = u.render(cams, 1.0, 1, **ALL)
    first = u.instance_first
    for w, (width, height, insts) in enumerate(worlds):
        plain = ng.BatchRenderer(width, height, 1, 1, [], lights, floor, new, insts, device="cuda:0")
        if insts:
            plain.set_instance_transforms(mats[first[w]:first[w + 1]].reshape(1, len(insts), 3, 4))
        mine = {k: u.image(v, w)[None] for k, v in got.items()}
        P.assert_same_images(mine, plain.render(cams[w:w + 1], 1.0, 1, **ALL), rgb_tol=0)
