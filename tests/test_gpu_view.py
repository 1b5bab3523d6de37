"""The single-view Renderer (ngb_render_view, ngb_render_view_frame; neraulgraphics_b200.Renderer) against the
oracle's restatement of the reference's Renderer (the running average of render_pixel, src/render_core.h:288-301)
and against the reference's own Renderer on its CPU backend.

The picture of frame k > 0 averages its samples with the frames before it, so a pixel whose rays met a near tie
(two hits within 1e-6 relative t, flagged by the oracle) in any frame so far is exempt; elsewhere the ARGB bytes
are within one level (CUDA's sinf, cosf and powf against the host's) and depth, normals and IDs bit-exact. The
scenes cover every kernel the view render runs: the per-pixel kernel (a mirror sphere, two lights, two samples
per frame), the tile kernels (eight icospheres, one soft-shadow light) and, for the world of 100,000 instances,
the warp-packet walk with the shadow rays as persistent-kernel jobs.
"""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
import scenes
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu
FRAMES = ((0, 1), (1, 2), (2, 1), (0, 2), (1, 1))


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def channels(argb):
    return np.stack([(argb >> 16) & 0xFF, (argb >> 8) & 0xFF, argb & 0xFF], -1).astype(int)


def view_scenes():
    t = scenes.template(worlds=1)
    wl = workloads.icosphere_worlds(worlds=1, width=80, height=60, seed=5)
    return [("template", t, scenes.template_matrices(1),
             ng.make_camera((0.3, 0.6, 0.2), (0, 0, -8), width=t.width, height=t.height, fov=scenes.FOV)),
            ("icospheres", wl.desc, wl.matrices, ng.make_camera((0.1, 1.1, 0.1), (0, 0, -6), width=80, height=60,
                                                               fov=1.0))]


def renderer(d, mats):
    r = ng.Renderer(d.width, d.height, d.spheres, d.lights, d.floor, d.meshes, d.instances, device="cuda:0")
    r.set_instance_transforms(np.asarray(mats, np.float32).reshape(-1, 3, 4))
    return r


@pytest.mark.parametrize("kernel", [0, 1])
def test_view_render_averages_frames_like_the_oracle_and_the_reference(torch_cuda, kernel):
    for name, d, mats, cam in view_scenes():
        r = renderer(d, mats)
        r.set_tuning(kernel=kernel)
        o, ref = O.Oracle(d), O.ReferenceView(d)
        o.set_instance_transforms(mats)
        ref.set_instance_transforms(mats)
        tie = None
        for frame, spp in FRAMES:
            got = r.render_argb(cam, frame, spp)
            want = o.render_view(cam, frame, spp, rgb=True, ties=True)
            flags = want["ties"] != 0
            tie = flags if frame == 0 else (tie | flags)
            theirs = ref.render(cam, frame, spp)
            assert (got >> 24 == 0xFF).all()
            for other, what in ((want["argb"], "oracle"), (theirs, "reference")):
                off = np.abs(channels(got) - channels(other)).max(-1)[~tie]
                assert off.max(initial=0) <= 1, f"{name} frame {frame} spp {spp}: {what} {off.max()} levels"
            print(f"\n{name} kernel {kernel} frame {frame} spp {spp}: near-tie pixels so far {int(tie.sum())}")
        # render() is the same picture as RGB bytes.
        rgb = r.render(cam, 3, 1)
        want = o.render_view(cam, 3, 1, rgb=True, ties=True)
        tie |= want["ties"] != 0
        assert np.abs(rgb.astype(int) - channels(want["argb"])).max(-1)[~tie].max(initial=0) <= 1


def test_view_render_frame_images(torch_cuda):
    """render_frame: depth, normals and IDs bit for bit off near ties; its RGB is the running average's bytes,
    which it advances as render does; zero-copy CUDA tensors alias the renderer's buffers."""
    torch = torch_cuda
    for name, d, mats, cam in view_scenes():
        r, o = renderer(d, mats), O.Oracle(d)
        o.set_instance_transforms(mats)
        tie = None
        for frame, spp in FRAMES:
            got = r.render_frame(cam, frame, spp, rgb=True, depth=True, normals=True, object_ids=True)
            want = o.render_view(cam, frame, spp, rgb=True, depth=True, normals=True, object_ids=True, ties=True)
            flags = want["ties"] != 0
            tie = flags if frame == 0 else (tie | flags)
            ok = (want["ties"] & (O.TIE_AOV_INSTANCE | O.TIE_AOV_TRIANGLE)) == 0
            assert np.array_equal(got["object_ids"][ok], want["object_ids"][ok]), name
            assert np.array_equal(bits(got["depth"][ok]), bits(want["depth"][ok])), name
            assert np.array_equal(bits(got["normals"][ok]), bits(want["normals"][ok])), name
            off = np.abs(got["rgb"].astype(int) - channels(want["argb"])).max(-1)[~tie]
            assert off.max(initial=0) <= 1, f"{name} frame {frame}: {off.max()} levels"
        dev = r.render_frame(cam, 0, 1, rgb=False, depth=True, object_ids=True, zero_copy=True)
        assert dev["depth"].is_cuda and tuple(dev["depth"].shape) == (d.height, d.width)
        host = r.render_frame(cam, 0, 1, rgb=False, depth=True, object_ids=True)
        assert np.array_equal(dev["object_ids"].cpu().numpy(), host["object_ids"])
        torch.cuda.synchronize()


def test_view_of_100000_instances_at_1280x720(torch_cuda):
    """The large world through the single-view entry: the frame's images and a LiDAR sweep (cast_rays of (N, 3)
    rays) against the oracle."""
    wl = workloads.large_world()
    d = wl.desc
    cam = ng.make_camera((0.0, 2.0, -100.0), (0.0, 0.0, 0.0), width=d.width, height=d.height, fov=1.0)
    r, o = renderer(d, wl.matrices[0]), O.Oracle(d)
    o.set_instance_transforms(wl.matrices[0])
    got = r.render_frame(cam, 0, 1, rgb=True, depth=True, object_ids=True)
    want = o.render_view(cam, 0, 1, rgb=True, depth=True, object_ids=True, ties=True)
    aov = (want["ties"] & O.TIE_AOV_INSTANCE) == 0
    pic = (want["ties"] & O.TIE_RGB_INSTANCE) == 0
    assert (want["object_ids"] >= ng.OBJECT_INSTANCE).mean() > 0.5
    assert np.array_equal(got["object_ids"][aov], want["object_ids"][aov])
    assert np.array_equal(bits(got["depth"][aov]), bits(want["depth"][aov]))
    off = np.abs(got["rgb"].astype(int) - channels(want["argb"])).max(-1)[pic]
    assert off.max(initial=0) <= 1
    ties = int((want["ties"] != 0).sum())
    print(f"\nview 1280x720, 100,000 instances: near-tie pixels {ties}, RGB one level off {int((off > 0).sum())}")
    assert ties <= 1e-4 * want["ties"].size
    lidar = wl.info["lidar"]
    hits = r.cast_rays(lidar["origins"][0], lidar["directions"][0], lidar["max_distance"])
    exp = o.cast_rays(lidar["origins"], lidar["directions"], lidar["max_distance"])
    assert hits["distance"].shape == (lidar["origins"].shape[1],)
    for k in ("object_id", "distance", "normal"):
        assert np.array_equal(bits(hits[k]), bits(exp[k][0])), k


def test_view_checks_its_arguments(torch_cuda):
    name, d, mats, cam = view_scenes()[1]
    r = renderer(d, mats)
    with pytest.raises(ValueError, match="frame must be 0 or more"):
        r.render(cam, -1, 1)
    with pytest.raises(ValueError, match="samples_per_frame must be 1 or more"):
        r.render(cam, 0, 0)
    bad = ng.Camera(cam.position, cam.right, cam.up, (float("nan"), 0.0, -1.0), cam.fov_scale, cam.aspect)
    with pytest.raises(ValueError, match="camera has a NaN or infinite value"):
        r.render(bad, 0, 1)
    with pytest.raises(ValueError, match="render_frame needs at least one output"):
        r.render_frame(cam, 0, 1, rgb=False)
    batch = ng.BatchRenderer(d.width, d.height, 2, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                             device="cuda:0")
    import ctypes as C
    from neraulgraphics_b200.renderer import _camera_c
    argb = np.zeros((d.height, d.width), np.uint32)
    status = batch._lib.ngb_render_view(batch._h, C.byref(_camera_c(cam)), 0, 1, argb.ctypes.data_as(C.c_void_p))
    assert status == 1  # NGB_INVALID_ARGUMENT
    assert "one world seen by one camera" in batch._lib.ngb_last_error(batch._h).decode()
