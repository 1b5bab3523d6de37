"""CPU tests: the oracle is pinned to the reference (golden fixtures made by the reference itself, and the
reference library when it is built here), and the product's host pieces match the reference bit-exactly."""

import os
import re

import numpy as np
import pytest

import oracle as O
from neraulgraphics_b200 import scene as S, workloads
import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref/libngref.so is not built")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def assert_images_equal(got, want, rgb_tol=0):
    for k in ("object_ids", "depth", "normals"):
        if k in want and k in got:
            assert np.array_equal(bits(got[k]) if got[k].dtype == np.float32 else got[k],
                                  bits(want[k]) if want[k].dtype == np.float32 else want[k]), k
    if "rgb" in want and "rgb" in got:
        d = np.abs(got["rgb"].astype(int) - want["rgb"].astype(int))
        assert d.max() <= rgb_tol, f"rgb differs by {d.max()}"


# ------------------------------------------------------------------------------- oracle vs golden --

def test_oracle_matches_reference_fixture_icospheres():
    f = np.load(os.path.join(GOLDEN, "icosphere_16x8_seed0.npz"))
    wl = workloads.icosphere_worlds(worlds=16, per_world=8, seed=0)
    assert np.array_equal(wl.matrices, f["matrices"]) and np.array_equal(wl.cameras, f["cameras"])
    o = O.Oracle(wl.desc)
    o.set_instance_transforms(f["matrices"])
    got = o.render(f["cameras"], float(f["fov"]), 1, rgb=True, depth=True, normals=True, object_ids=True)
    assert_images_equal(got, f)
    assert (f["object_ids"] >= S._abi.OBJECT_INSTANCE).mean() > 0.05


def test_oracle_matches_reference_fixture_template():
    """Spheres, a mirror (reflection bounces), two hard-shadow lights, a checker floor, smooth normals,
    ambient 0.1, 2 samples per pixel, frame 5."""
    f = np.load(os.path.join(GOLDEN, "template_6w_spp2_frame5.npz"))
    o = O.Oracle(scenes.template(worlds=6))
    o.set_instance_transforms(f["matrices"])
    o.set_ambient(float(f["ambient"]))
    got = o.render(f["cameras"], float(f["fov"]), 2, rgb=True, depth=True, normals=True, object_ids=True, frame=5)
    assert_images_equal(got, f)


def test_oracle_matches_reference_fixture_bodies_and_rays():
    f = np.load(os.path.join(GOLDEN, "body_16x20_seed0.npz"))
    wl = workloads.body_worlds(worlds=16, seed=0)
    o = O.Oracle(wl.desc)
    o.bind_bodies(**wl.binding)
    o.set_body_poses(f["poses"])
    assert np.array_equal(bits(o.tlas()["matrices"].reshape(f["matrices"].shape)), bits(f["matrices"]))
    got = o.render(f["cameras"], float(f["fov"]), 1, rgb=True, depth=True, object_ids=True)
    assert_images_equal(got, f)
    hits = o.cast_rays(f["ray_origins"], f["ray_directions"], 20.0)
    assert np.array_equal(hits["object_id"], f["ray_object_id"])
    assert np.array_equal(bits(hits["distance"]), bits(f["ray_distance"]))
    assert np.array_equal(bits(hits["normal"]), bits(f["ray_normal"]))


# --------------------------------------------------------------------------- known answers (oracle) --

def test_oracle_known_answers():
    desc, mats, cams = scenes.one_box_worlds()
    o = O.Oracle(desc)
    o.set_instance_transforms(mats)
    d = o.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[:, scenes.H // 2, scenes.W // 2] == pytest.approx([7.0, 2.0], abs=0.02)
    hits = o.cast_rays(np.zeros((2, 1, 3), np.float32), np.tile(np.float32([0, 0, -1]), (2, 1, 1)), 100.0)
    assert hits["distance"][:, 0] == pytest.approx([7.0, 2.0], abs=1e-3)
    assert (hits["object_id"] == S._abi.OBJECT_INSTANCE).all()
    desc, mats, cams = scenes.single_leaf_worlds()
    o = O.Oracle(desc)
    o.set_instance_transforms(mats)
    d = o.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[:, scenes.H // 2, scenes.W // 2] == pytest.approx([3.0, 4.0, 5.0, 6.0], abs=0.02)
    desc, mats, cams = scenes.coincident_boxes()
    o = O.Oracle(desc)
    o.set_instance_transforms(mats)
    d = o.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[0, scenes.H // 2, scenes.W // 2] == pytest.approx(4.8, abs=0.02)


def test_oracle_lbvh_structure():
    """Every world's tree reaches each of its leaves once, links are consistent and boxes contain children."""
    desc, mats, cams = scenes.scattered_boxes(30, 40)
    o = O.Oracle(desc)
    o.set_instance_transforms(mats)
    t = o.tlas()
    nodes, roots, n = t["nodes"], t["roots"], 30 * 40
    lo = nodes[:, :3].view(np.float32)
    hi = nodes[:, 4:7].view(np.float32)
    for w in range(30):
        seen, stack = [], [roots[w]]
        while stack:
            v = stack.pop()
            left, right = nodes[v, 3], nodes[v, 7]
            if left < 0:
                seen.append(~left)
                continue
            for c in (left, right):
                assert (lo[v] <= lo[c]).all() and (hi[v] >= hi[c]).all()
                stack.append(c)
        assert sorted(seen) == list(range(w * 40, (w + 1) * 40))
    assert sorted(t["sorted_ids"]) == list(range(n))
    keys = t["keys"][t["sorted_ids"]]
    assert (np.diff(keys.astype(np.float64)) >= 0).all()


# ------------------------------------------------------------------- host pieces vs the reference --

@needs_ref
@pytest.mark.parametrize("radius,sub", [(0.5, 2), (0.5, 3), (1.0, 1), (2.0, 4)])
def test_icosphere_generator_is_the_references(radius, sub):
    a, b = S.make_icosphere(radius, sub), O.ref_make_icosphere(radius, sub)
    assert np.array_equal(bits(a.vertices), bits(b.vertices)) and np.array_equal(a.triangles, b.triangles)


@needs_ref
def test_transform_and_box_generators_are_the_references():
    rng = np.random.default_rng(0)
    for _ in range(500):
        p, q, s = rng.uniform(-3, 3, 3), rng.normal(size=4), rng.uniform(0.2, 2)
        assert np.array_equal(bits(S.make_transform(p, q, s).matrix), bits(O.ref_make_transform(p, q, s)))
    a, b = S.make_box((0.4, 0.5, 0.6)), O.ref_make_box((0.4, 0.5, 0.6))
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.triangles, b.triangles)
    m = S.make_camera((0.1, 1.2, 0.3), (0, 0, -6), width=64, height=48, fov=1.0).matrix
    assert np.array_equal(bits(m), bits(O.ref_camera_matrix((0.1, 1.2, 0.3), (0, 0, -6), (0, 1, 0), 1.0, 64, 48)))


@needs_ref
def test_blas_builders_are_the_references():
    """The product's host builder (libngb.so) and the oracle's both give the reference's trees bit for bit."""
    import neraulgraphics_b200 as ng
    smooth = S.make_icosphere(1.0, 2)
    rng = np.random.default_rng(5)
    soup = S.Mesh(rng.normal(size=(600, 3)).astype(np.float32), np.arange(600, dtype=np.uint32).reshape(200, 3))
    same = S.Mesh(np.tile(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), (10, 1)),
                  np.arange(30, dtype=np.uint32).reshape(10, 3))
    one = S.Mesh(np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0]]), np.uint32([[0, 1, 2]]))
    zeros = S.Mesh(np.float32([[0, 0, 0], [-0.0, 1, 0], [0, -0.0, 1], [1, 1, -0.0], [-0.0, -0.0, -0.0]]),
                   np.uint32([[0, 1, 2], [1, 3, 4], [4, 2, 0], [3, 2, 1]]))
    line = S.Mesh(np.float32([[i, 0, 0] for i in range(40)] + [[i, 1e-3, 0] for i in range(40)]),
                  np.uint32([[i, i + 1, 40 + i] for i in range(39)]))
    meshes = [S.make_icosphere(0.5, 3), S.make_box((0.4, 0.4, 0.4)), S.cylinder(1.0, 1.0, 128),
              S.Mesh(smooth.vertices, smooth.triangles, normals=smooth.vertices), S.make_icosphere(1.0, 5),
              soup, same, one, zeros, line]
    want = O.ref_build_meshes(meshes)
    got = ng.build_meshes(meshes)
    inst = [S.Instance(i) for i in range(len(meshes))]
    orc = O.Oracle(S.SceneDesc(8, 8, 1, meshes=meshes, instances=inst)).blas()
    for k in ("nodes", "triangles", "roots", "bounds"):
        w = bits(want[k]) if want[k].dtype == np.float32 else want[k]
        for g in (got, orc):
            x = bits(g[k]) if g[k].dtype == np.float32 else g[k]
            assert np.array_equal(x, w), k
    assert np.array_equal(got["triangle_index"], orc["triangle_index"])


@needs_ref
def test_oracle_compose_against_reference_double_compose():
    """The single-precision compose (the reference's GPU path) is within float rounding of its host twin
    (double precision, src/instances.cpp:137-164)."""
    wl = workloads.body_worlds(worlds=8)
    b = wl.binding
    m32 = O.compose(8, 20, 20, b["body_of_instance"], b["local_pose"], b["scale"], wl.poses)
    m64 = O.ref_body_poses_to_matrices(b["body_of_instance"], b["local_pose"], b["scale"], 20, 8, wl.poses)
    assert np.abs(m32 - m64).max() <= 1e-6 * max(1.0, np.abs(m64).max())


@needs_ref
def test_oracle_matches_reference_on_scattered_worlds_except_near_ties():
    desc, mats, cams = scenes.scattered_boxes(50, 40)
    o, r = O.Oracle(desc), O.Reference(desc)
    o.set_instance_transforms(mats)
    r.set_instance_transforms(mats)
    a = o.render(cams, scenes.FOV, 1, rgb=True, depth=True, normals=True, object_ids=True, ties=True)
    b = r.render(cams, scenes.FOV, 1, rgb=True, depth=True, normals=True, object_ids=True)
    tie = (a["ties"] & O.TIE_AOV_INSTANCE) != 0
    assert ((a["object_ids"] != b["object_ids"]) & ~tie).sum() == 0
    same = (a["object_ids"] == b["object_ids"]) & ~tie
    assert np.array_equal(bits(a["depth"][same]), bits(b["depth"][same]))
    rgb_tie = (a["ties"] & O.TIE_RGB_INSTANCE) != 0
    assert (np.abs(a["rgb"].astype(int) - b["rgb"].astype(int)).max(-1)[~rgb_tie] == 0).all()


def view_scenes():
    """Single-view scenes: the template (mirror sphere, two hard-shadow lights, checker floor, smooth normals) and
    eight icospheres under one soft-shadow light, each with its camera (make_camera)."""
    t = scenes.template(worlds=1)
    wl = workloads.icosphere_worlds(worlds=1, width=80, height=60, seed=5)
    return [(t, scenes.template_matrices(1), S.make_camera((0.3, 0.6, 0.2), (0, 0, -8), width=t.width,
                                                            height=t.height, fov=scenes.FOV)),
            (wl.desc, wl.matrices, S.make_camera((0.1, 1.1, 0.1), (0, 0, -6), width=80, height=60, fov=1.0))]


@needs_ref
def test_oracle_view_renders_are_the_references_renderer():
    """The oracle's single-view render (the running average over frames, and render_frame's images) against the
    reference's own Renderer on its CPU backend, frame after frame: ARGB, RGB, depth, normals and IDs bit for bit
    but on near ties (the reference's CPU backend builds its instance tree by SAH, the oracle by LBVH)."""
    for desc, mats, cam in view_scenes():
        o, r = O.Oracle(desc), O.ReferenceView(desc)
        o.set_instance_transforms(mats)
        r.set_instance_transforms(mats)
        tie = np.zeros((desc.height, desc.width), bool)
        for frame, spp in ((0, 1), (1, 2), (2, 1), (0, 2), (1, 1)):
            got = o.render_view(cam, frame, spp, rgb=True, depth=True, normals=True, object_ids=True, ties=True)
            want_argb = r.render(cam, frame, spp)
            tie = (tie | (got["ties"] != 0)) if frame else (got["ties"] != 0)
            assert np.array_equal(got["argb"][~tie], want_argb[~tie]), (frame, spp)
            assert (got["argb"] >> 24 == 0xFF).all()
            rgb = np.stack([(got["argb"] >> 16) & 0xFF, (got["argb"] >> 8) & 0xFF, got["argb"] & 0xFF], -1)
            assert np.array_equal(rgb.astype(np.uint8), got["rgb"])
            want = r.render_frame(cam, frame + 1, spp, rgb=False, depth=True, normals=True, object_ids=True)
            ok = ~tie
            assert np.array_equal(got["object_ids"][ok], want["object_ids"][ok])
            assert np.array_equal(bits(got["depth"][ok]), bits(want["depth"][ok]))
            assert np.array_equal(bits(got["normals"][ok]), bits(want["normals"][ok]))


@needs_ref
def test_make_camera_is_the_references():
    """ngb_make_camera (the C ABI) and the Python make_camera against the reference's make_camera, every field."""
    import ctypes as C
    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import _abi
    from neraulgraphics_b200._lib import lib
    L = lib()
    rng = np.random.default_rng(4)
    for _ in range(300):
        p, t = rng.uniform(-5, 5, 3).astype(np.float32), rng.uniform(-5, 5, 3).astype(np.float32)
        fov, w, h = float(np.float32(rng.uniform(0.3, 2.0))), int(rng.integers(8, 300)), int(rng.integers(8, 300))
        want = O.ref_make_camera(p, t, (0, 1, 0), fov, w, h)
        c = _abi.CameraC()
        v = lambda a: _abi.Vec3(*[float(x) for x in a])
        assert L.ngb_make_camera(v(p), v(t), v((0, 1, 0)), fov, w, h, C.byref(c)) == 0
        got = np.float32([c.position.x, c.position.y, c.position.z, c.right.x, c.right.y, c.right.z, c.up.x, c.up.y,
                          c.up.z, c.forward.x, c.forward.y, c.forward.z, c.fov_scale, c.aspect])
        py = ng.make_camera(p, t, width=w, height=h, fov=fov)
        mine = np.float32(list(py.position) + list(py.right) + list(py.up) + list(py.forward) + [py.fov_scale,
                                                                                                py.aspect])
        assert np.array_equal(bits(got), bits(want)) and np.array_equal(bits(mine), bits(want))


# ----------------------------------------------------------------------------------------- the ABI --

def test_library_exports_every_declared_entry_point():
    import ctypes
    header = open(os.path.join(ROOT, "include", "ngb.h")).read()
    declared = sorted(set(re.findall(r"^\w[\w\s\*]*?\b(ngb_\w+)\(", header, re.M)))
    assert len(declared) >= 28
    lib = ctypes.CDLL(os.path.join(ROOT, "neraulgraphics_b200", "libngb.so"))
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing


def test_stream_entry_points_check_their_arguments_before_any_launch():
    """The handle-free entry points (pose matrices, their gradient) reject bad arguments on the host, with a
    message in ngb_last_error(NULL), and do nothing for zero poses; no GPU is touched."""
    import ctypes
    from neraulgraphics_b200._lib import lib
    L = lib()
    L.ngb_last_error.restype = ctypes.c_char_p
    assert L.ngb_pose_matrices(None, None, None, 0, None, None) == 0
    assert L.ngb_pose_matrices(None, None, None, 5, None, None) == 1
    assert b"positions, quaternions and matrices must not be null" in L.ngb_last_error(None)
    assert L.ngb_pose_matrices(None, None, None, -1, None, None) == 1
    assert L.ngb_pose_matrices_grad(None, None, 0, None, None, None, None, None) == 0
    assert L.ngb_pose_matrices_grad(None, None, 3, None, None, None, None, None) == 1
    dummy = ctypes.c_void_p(16)
    assert L.ngb_pose_matrices_grad(dummy, None, 3, dummy, dummy, dummy, dummy, None) == 1
    assert b"grad_scales needs scales" in L.ngb_last_error(None)


def test_row_band_and_memory_entry_points_without_a_renderer():
    """ngb_set_rows on no renderer is a logic error, ngb_rows checks its pointers, and with no renderer made the
    device-bytes count is 0, also after a construction that validation refused (its cleanup touches no GPU)."""
    import ctypes
    import neraulgraphics_b200 as ng
    from neraulgraphics_b200._lib import lib
    L = lib()
    assert L.ngb_set_rows(None, 0, 1) == 4
    first, count = ctypes.c_int32(), ctypes.c_int32()
    assert L.ngb_rows(None, ctypes.byref(first), ctypes.byref(count)) == 1
    assert L.ngb_inject_allocation_failure(-1) == 0
    assert ng.device_bytes() == 0
    with pytest.raises(ValueError, match="world_count must be 1 or more"):
        ng.BatchRenderer(8, 8, 0, 1)
    assert ng.device_bytes() == 0


def test_construction_rejects_bad_scenes_with_the_reference_messages():
    import neraulgraphics_b200 as ng
    with pytest.raises(ValueError, match="world_count must be 1 or more, got 0"):
        ng.BatchRenderer(64, 64, 0)
    with pytest.raises(ValueError, match="cameras_per_world must be 1 or more, got 0"):
        ng.BatchRenderer(64, 64, 1, 0)
    with pytest.raises(ValueError, match="frame size must be positive, got 0x64"):
        ng.BatchRenderer(0, 64, 1)
    with pytest.raises(ValueError, match="instance 0 uses mesh 2, but there are 1 meshes"):
        ng.BatchRenderer(64, 64, 1, meshes=[ng.make_box((1, 1, 1))], instances=[ng.Instance(2)])
    with pytest.raises(ValueError, match="instance 0 transform is singular"):
        ng.BatchRenderer(64, 64, 1, meshes=[ng.make_box((1, 1, 1))],
                         instances=[ng.Instance(0, ng.Transform(np.zeros((3, 4), np.float32)))])
    with pytest.raises(ValueError, match="light 0 radius must be 0 or more"):
        ng.BatchRenderer(64, 64, 1, lights=[ng.Light((0, 1, 0), 1.0, -1.0)])
    with pytest.raises(ValueError, match="scene has 9 lights, at most 8 fit"):
        ng.BatchRenderer(64, 64, 1, lights=[ng.Light((0, 1, 0))] * 9)
    with pytest.raises(ValueError, match="mesh 0 index 2 is 7, but there are only 3 vertices"):
        ng.BatchRenderer(64, 64, 1, meshes=[ng.Mesh(np.zeros((3, 3)), [[0, 1, 7]])], instances=[ng.Instance(0)])
    with pytest.raises(ValueError, match="device 'cpu' is not available"):
        ng.BatchRenderer(64, 64, 1, device="cpu")


def test_workloads_are_deterministic():
    a, b = workloads.body_worlds(worlds=4, seed=3), workloads.body_worlds(worlds=4, seed=3)
    assert np.array_equal(a.poses, b.poses) and np.array_equal(a.cameras, b.cameras)
    s1 = workloads.random_walk(a.poses, 3, seed=1)
    s2 = workloads.random_walk(b.poses, 3, seed=1)
    assert np.array_equal(s1, s2) and s1.shape == (3, 4, 20, 7)
    assert np.allclose(np.linalg.norm(s1[..., 3:], axis=-1), 1.0, atol=1e-6)


def test_srgb_threshold_table_reproduces_the_host_mapping_for_every_float():
    """The renderer turns linear light into sRGB bytes with a threshold table made on the host by bisection;
    an exhaustive scan of every float in [0, 1] (the oracle's srgb_channel, the reference's formula) shows the
    mapping never decreases and that the table's thresholds are exactly the first floats of each byte."""
    import ctypes
    from neraulgraphics_b200._lib import lib
    first = np.zeros(256, np.float32)
    L = O.oracle_lib()
    L.orc_srgb_scan.restype = ctypes.c_longlong
    L.orc_srgb_scan.argtypes = [ctypes.c_void_p]
    drops = L.orc_srgb_scan(first.ctypes.data_as(ctypes.c_void_p))
    assert drops == 0
    table = np.zeros(256, np.float32)
    assert lib().ngb_srgb_thresholds(table.ctypes.data_as(ctypes.c_void_p)) == 0
    assert np.array_equal(bits(table), bits(first))


def test_pose_matrices_agree_between_torch_and_numpy():
    """autodiff.pose_matrices (torch, differentiable) and workloads.pose_matrices_np make the same matrices."""
    import torch

    from neraulgraphics_b200.autodiff import pose_matrices
    wl = workloads.differentiable_worlds(worlds=3, width=16, height=16)
    i = wl.info
    t = pose_matrices(torch.from_numpy(i["positions"]), torch.from_numpy(i["quaternions"]), torch.from_numpy(i["scales"]))
    assert np.abs(t.numpy() - wl.matrices).max() <= 1e-6
    q = torch.from_numpy(i["quaternions"][0, :2]).double().requires_grad_()
    p = torch.from_numpy(i["positions"][0, :2]).double()
    assert torch.autograd.gradcheck(lambda qq: pose_matrices(p, qq), (q,))


def test_geom_matrices_are_the_compose_kernels_products():
    """O.geom_matrices against a plain loop of the compose kernel's float32 products (mujoco.py:291-302)."""
    rng = np.random.default_rng(0)
    xpos = rng.normal(size=(3, 5, 3)).astype(np.float32)
    xmat = rng.normal(size=(3, 5, 3, 3)).astype(np.float32)
    goi = np.int32([4, 0, 2])
    scale = rng.uniform(0.1, 2.0, size=(3, 3)).astype(np.float32)
    got = O.geom_matrices(xpos, xmat, goi, scale)
    for w in range(3):
        for i, g in enumerate(goi):
            for row in range(3):
                for c in range(3):
                    assert got[w, i, row, c] == np.float32(xmat[w, g, row, c] * scale[i, c])
                assert got[w, i, row, 3] == xpos[w, g, row]
