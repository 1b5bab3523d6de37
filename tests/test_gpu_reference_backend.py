"""The boundary proved from the reference's side: the reference's own BatchRenderer and Renderer (neraulgraphics
0.5.0, compiled from its sources) drawing through this library, with oracle/ngb_backend.cpp as their CUDA backend
(the reference's backend seam, src/backend.h:36-88, implemented on include/ngb.h).

  - the reference's known answers (tests/test_batch.cpp:183-208, 307-331): worlds see only their own instances,
    single-leaf trees, a thousand coincident boxes, and ray queries per world;
  - the reference's body-pose case (tests/test_batch.cpp:210-269): bodies with offsets and scales give the picture
    of the matrices worked out by hand, to 1 object-ID pixel in 5000;
  - the reference's classes and this library's own give the same images bit for bit on the same inputs (one
    implementation under two fronts), for a batch of bodies and for a single view over several frames.
"""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
import scenes
from neraulgraphics_b200 import workloads

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.reference_available(ngb=True),
                                 reason="oracle/_ref/libngref_ngb.so is not built (make -C oracle ref-ngb)")]
ALL = dict(rgb=True, depth=True, normals=True, object_ids=True)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_reference_known_answers_through_this_library(torch_cuda):
    desc, mats, cams = scenes.one_box_worlds()
    r = O.Reference(desc, ngb=True)
    r.set_instance_transforms(mats)
    d = r.render(cams, scenes.FOV, 1, rgb=False, depth=True, object_ids=True)["depth"]
    assert d[:, scenes.H // 2, scenes.W // 2] == pytest.approx([7.0, 2.0], abs=0.02)
    hits = r.cast_rays(np.zeros((2, 1, 3), np.float32), np.tile(np.float32([0, 0, -1]), (2, 1, 1)), 100.0)
    assert hits["distance"][:, 0] == pytest.approx([7.0, 2.0], abs=1e-3)
    assert (hits["object_id"] == ng.OBJECT_INSTANCE).all()
    desc, mats, cams = scenes.single_leaf_worlds()
    r = O.Reference(desc, ngb=True)
    r.set_instance_transforms(mats)
    d = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[:, scenes.H // 2, scenes.W // 2] == pytest.approx([3.0, 4.0, 5.0, 6.0], abs=0.02)
    desc, mats, cams = scenes.coincident_boxes()
    r = O.Reference(desc, ngb=True)
    r.set_instance_transforms(mats)
    d = r.render(cams, scenes.FOV, 1, rgb=False, depth=True)["depth"]
    assert d[0, scenes.H // 2, scenes.W // 2] == pytest.approx(4.8, abs=0.02)


def quaternion_matrix(q):
    x, y, z, w = (np.float32(v) for v in q)
    return np.float32([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                       [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                       [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def test_reference_body_poses_through_this_library_equal_hand_matrices(torch_cuda):
    """Two bodies per world and three instances, one on each body with an offset and a scale, one fixed."""
    worlds = 4
    desc = scenes.template(worlds=worlds)
    boi = np.int32([0, 1, -1])
    local = np.float32([[0.5, 0, 0, 0, 0, 0, 1], [0, 0.4, 0, 0, 0.3826834, 0, 0.9238795], [2, 0, -7, 0, 0, 0, 1]])
    scale = np.float32([[1, 1, 1], [0.5, 0.5, 1.0], [1, 1, 1]])
    rng = np.random.default_rng(11)
    bodies = np.float32([[[-1.5 + 3.0 * k + 0.2 * w, 0.0, -6.0 - rng.random(), 0.0, 0.2588190 * (1 if k else -1),
                           0.0, 0.9659258] for k in range(2)] for w in range(worlds)])
    b = O.Reference(desc, ngb=True)
    b.bind_bodies(boi, local, scale, 2)
    b.set_body_poses(bodies)
    mats = np.zeros((worlds, 3, 3, 4), np.float32)
    for w in range(worlds):
        for i in range(3):
            rl = quaternion_matrix(local[i, 3:])
            r, p = rl, local[i, :3].copy()
            if boi[i] >= 0:
                bp = bodies[w, boi[i]]
                rb = quaternion_matrix(bp[3:])
                r = (rb @ rl).astype(np.float32)
                p = (bp[:3] + rb @ local[i, :3]).astype(np.float32)
            mats[w, i, :, :3] = r * scale[i][None, :]
            mats[w, i, :, 3] = p
    m = O.Reference(desc, ngb=True)
    m.set_instance_transforms(mats)
    cams = np.stack([scenes.camera((0, 0.5, 0), (0, 0, -8))] * worlds)
    a, c = b.render(cams, scenes.FOV, 1, **ALL), m.render(cams, scenes.FOV, 1, **ALL)
    diff = int((a["object_ids"] != c["object_ids"]).sum())
    print(f"\nbody poses vs hand matrices through the reference's BatchRenderer on this library: {diff} ID pixels")
    assert diff <= a["object_ids"].size // 5000
    assert (a["object_ids"] == ng.OBJECT_INSTANCE + 1).any()


def test_reference_classes_draw_this_librarys_images(torch_cuda):
    wl = workloads.body_worlds(worlds=64, seed=3)
    d = wl.desc
    ref = O.Reference(d, ngb=True)
    mine = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                            device="cuda:0")
    for x in (ref, mine):
        x.bind_bodies(**wl.binding)
    for step in workloads.random_walk(wl.poses, 2, seed=4):
        ref.set_body_poses(step)
        mine.set_body_poses(step)
        a = ref.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=1)
        b = mine.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=1)
        for k in a:
            assert np.array_equal(np.ascontiguousarray(a[k]).view(np.uint8), np.ascontiguousarray(b[k]).view(np.uint8)), k
    # The single-view Renderer: the running average over frames, render_frame's images and ray queries.
    wl = workloads.icosphere_worlds(worlds=1, width=80, height=60, seed=2)
    cam = ng.make_camera((0.2, 1.0, 0.1), (0, 0, -6), width=80, height=60, fov=1.0)
    view = O.ReferenceView(wl.desc, ngb=True)
    own = ng.Renderer(80, 60, wl.desc.spheres, wl.desc.lights, wl.desc.floor, wl.desc.meshes, wl.desc.instances,
                      device="cuda:0")
    view.set_instance_transforms(wl.matrices)
    own.set_instance_transforms(wl.matrices.reshape(-1, 3, 4))
    for frame, spp in ((0, 1), (1, 2), (2, 1)):
        assert np.array_equal(view.render(cam, frame, spp), own.render_argb(cam, frame, spp)), frame
    a = view.render_frame(cam, 0, 1, **ALL)
    b = own.render_frame(cam, 0, 1, **ALL)
    for k in a:
        assert np.array_equal(np.ascontiguousarray(a[k]).view(np.uint8), np.ascontiguousarray(b[k]).view(np.uint8)), k
