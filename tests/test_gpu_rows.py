"""Row bands (BatchRenderer.set_rows, ngb_set_rows): a renderer that draws rows [first, first + count) of every
view gives exactly those rows of the whole image, bit for bit, on every render kernel (the per-pixel kernel,
the persistent kernel, the tile kernels with candidate lists of 32 and 256 and the packet walk); the hit
records and the depth/normal adjoint of a band are the whole image's restricted to it; one rank's
ShardedFrame round trip is the whole image."""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
from neraulgraphics_b200 import workloads
from neraulgraphics_b200.sharding import ShardedFrame

pytestmark = pytest.mark.gpu
ALL = dict(rgb=True, depth=True, normals=True, object_ids=True)
# Bands of a 29-row image: the first row, a band across tile edges, one ending at the last row, the last row.
BANDS = [(0, 1), (5, 7), (13, 16), (28, 1)]


def renderer(d):
    return ng.BatchRenderer(d.width, d.height, d.world_count, d.cameras_per_world, d.spheres, d.lights, d.floor,
                            d.meshes, d.instances, device="cuda:0")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8) if a.dtype == np.uint8 else a.view(np.uint32)


# (instances per world, kernel and shape): candidate lists of 32 and 256, the packet walk; the persistent and
# per-pixel kernels; two samples per pixel (the per-pixel kernel, automatically).
CASES = [
    (8, dict(kernel=3, threads_per_block=128, registers=56), 1),
    (40, dict(kernel=3, threads_per_block=128, registers=56), 1),
    (300, dict(kernel=3, threads_per_block=128, registers=56), 1),
    (40, dict(kernel=2), 1),
    (300, dict(kernel=2), 1),
    (40, dict(kernel=1), 1),
    (8, dict(kernel=0), 2),
]


@pytest.mark.parametrize("per_world,tuning,spp", CASES)
def test_a_band_is_those_rows_of_the_whole_image(torch_cuda, per_world, tuning, spp):
    wl = workloads.icosphere_worlds(worlds=3, per_world=per_world, width=37, height=29, seed=29)
    d = wl.desc
    r = renderer(d)
    r.set_tuning(**tuning)
    r.set_instance_transforms(wl.matrices)
    want = r.render(wl.cameras, wl.fov, spp, **ALL, frame=3)
    assert (want["object_ids"] >= 34).mean() > 0.1
    assert r.rows == (0, 29)
    for first, count in BANDS:
        r.set_rows(first, count)
        assert r.rows == (first, count) and r.pixel_count == 3 * count * 37
        got = r.render(wl.cameras, wl.fov, spp, **ALL, frame=3)
        for k in want:
            assert got[k].shape == want[k][:, first:first + count].shape, k
            assert np.array_equal(bits(got[k]), bits(want[k][:, first:first + count])), (k, first, count)
    r.set_rows()
    assert r.rows == (0, 29)
    again = r.render(wl.cameras, wl.fov, spp, **ALL, frame=3)
    assert all(np.array_equal(bits(again[k]), bits(want[k])) for k in want)


def test_band_arguments_are_checked(torch_cuda):
    wl = workloads.icosphere_worlds(worlds=2, per_world=4, width=16, height=12, seed=1)
    r = renderer(wl.desc)
    for first, count in [(-1, 2), (0, 0), (11, 2), (12, 1), (0, 13)]:
        with pytest.raises(ValueError, match="rows"):
            r.set_rows(first, count)
    assert r.rows == (0, 12)
    d = wl.desc
    u = ng.UnevenBatchRenderer([(16, 12, d.instances[:2]), (8, 8, d.instances[:1])], lights=d.lights, floor=d.floor,
                               meshes=d.meshes, device="cuda:0")
    with pytest.raises(ValueError, match="uneven sizes render whole images"):
        u.set_rows(0, 4)


def test_band_hit_records_and_adjoint_are_the_whole_images_restricted(torch_cuda):
    """The adjoint over a band's pixels equals the whole image's adjoint with the gradient zero outside the band
    (float32 sums in another order: within 1e-5 relative)."""
    torch = torch_cuda
    from neraulgraphics_b200.autodiff import render_depth_normals
    wl = workloads.differentiable_worlds(worlds=3, width=40, height=29, seed=3)
    d = wl.desc
    first, count = 9, 13
    grads = []
    for band in (False, True):
        r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes,
                             d.instances, device="cuda:0")
        if band:
            r.set_rows(first, count)
        mats = torch.from_numpy(wl.matrices).cuda().requires_grad_()
        cams = torch.from_numpy(wl.cameras).cuda().requires_grad_()
        depth, normals = render_depth_normals(r, mats, cams, wl.fov)
        gen = torch.Generator(device="cuda").manual_seed(5)
        gd = torch.randn((3, 29, 40), device="cuda", generator=gen)
        gn = torch.randn((3, 29, 40, 3), device="cuda", generator=gen)
        gd, gn = gd[:, first:first + count], gn[:, first:first + count]
        if not band:
            depth, normals = depth[:, first:first + count], normals[:, first:first + count]
        finite = torch.isfinite(depth)
        loss = (torch.where(finite, depth, 0.0) * gd).sum() + (normals * gn).sum()
        loss.backward()
        hits = [torch.empty(depth.shape if band else (3, 29, 40), dtype=dt, device="cuda")
                for dt in (torch.int32, torch.int32, torch.float32, torch.float32)]
        r.record_hits(True)
        r.render(cams.detach(), wl.fov, 1, rgb=False, depth=True, normals=True, zero_copy=True)
        r.copy_hits(*hits)
        r.record_hits(False)
        if not band:
            hits = [h[:, first:first + count] for h in hits]
        grads.append((mats.grad.double().cpu().numpy(), cams.grad.double().cpu().numpy(),
                      [h.cpu().numpy() for h in hits], depth.detach().cpu().numpy()))
    (m0, c0, h0, d0), (m1, c1, h1, d1) = grads
    assert np.array_equal(bits(d0), bits(d1))
    assert all(np.array_equal(bits(a), bits(b)) for a, b in zip(h0, h1))
    assert (h0[0] >= 0).mean() > 0.1
    for a, b in ((m1, m0), (c1, c0)):
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), (np.linalg.norm(a - b), np.linalg.norm(b))


def test_sharded_frame_on_one_rank_is_the_whole_image(torch_cuda):
    torch = torch_cuda
    wl = workloads.icosphere_worlds(worlds=2, per_world=12, width=33, height=21, seed=7)
    r = renderer(wl.desc)
    r.set_instance_transforms(wl.matrices)
    want = {k: v.clone() for k, v in r.render(torch.from_numpy(wl.cameras).cuda(), wl.fov, 1, **ALL,
                                              zero_copy=True).items()}
    shard = ShardedFrame(height=21)
    assert (shard.first, shard.count) == (0, 21)
    shard.apply(r)
    got = r.render(torch.from_numpy(wl.cameras).cuda(), wl.fov, 1, **ALL, zero_copy=True)
    assert all(torch.equal(shard.gather(got[k]), want[k]) for k in want)
