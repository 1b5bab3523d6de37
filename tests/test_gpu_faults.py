"""Host-side fault injection (ngb_inject_allocation_failure): a device allocation that fails at any point of a
renderer's construction, a global tree build, a render, a ray query or a mesh rebuild raises CudaError; a
constructor frees everything it made (ngb_device_bytes back where it was), and a renderer keeps working: a
failed build leaves the previous tree in place, the same call made again gives what a renderer that never
failed gives, and nothing is left once the renderers are gone. The failure is made on the host in place of
cudaMalloc; no GPU fault is involved."""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu
ALL = dict(rgb=True, depth=True, normals=True, object_ids=True)


def scene():
    return workloads.icosphere_worlds(worlds=5, per_world=12, width=24, height=20, seed=4)


def make(d):
    return ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                            device="cuda:0")


def same(a, b):
    return all(np.array_equal(np.asarray(a[k]), np.asarray(b[k])) for k in a)


def until_it_works(call, limit=200, frees_all=False):
    """Fails the k-th allocation of call() for k = 0, 1, ... until call() makes fewer than k allocations; checks
    every failure's error and, with frees_all (a constructor), that it freed everything it made. Returns
    (call()'s result, the failures seen). A renderer's call keeps the arrays it made before the failing one:
    they are the renderer's, reused by the next call and freed with the renderer."""
    k = 0
    try:
        while True:
            before = ng.device_bytes()
            ng.inject_allocation_failure(k)
            try:
                out = call()
            except ng.CudaError as e:
                assert "out of memory" in str(e) and "injected" in str(e), str(e)
                if frees_all:
                    assert ng.device_bytes() == before
                k += 1
                assert k < limit
                continue
            return out, k
    finally:
        ng.inject_allocation_failure(-1)


def test_construction_that_fails_frees_everything(torch_cuda):
    wl = scene()
    base = ng.device_bytes()
    r, failures = until_it_works(lambda: make(wl.desc), frees_all=True)
    assert failures >= 10, failures      # the constructor's device arrays, each failed in turn
    assert ng.device_bytes() > base
    r.set_instance_transforms(wl.matrices)
    got = r.render(wl.cameras, wl.fov, 1, **ALL)
    clean = make(wl.desc)
    clean.set_instance_transforms(wl.matrices)
    assert same(got, clean.render(wl.cameras, wl.fov, 1, **ALL))
    del r, clean
    assert ng.device_bytes() == base


def test_failed_build_render_and_rays_leave_the_renderer_usable(torch_cuda):
    wl = scene()
    d = wl.desc
    base = ng.device_bytes()
    clean = make(d)
    clean.set_build(2)
    first = clean.render(wl.cameras, wl.fov, 1, **ALL)        # the tree of the instances' own transforms
    clean.set_instance_transforms(wl.matrices)
    want = clean.render(wl.cameras, wl.fov, 1, **ALL)
    rng = np.random.default_rng(2)
    origins = np.repeat(wl.cameras[:, None, :, 3], 64, axis=1).astype(np.float32)
    dirs = rng.normal(size=(5, 64, 3)).astype(np.float32)
    dirs[..., 2] = -np.abs(dirs[..., 2]) - 1.0
    want_rays = clean.cast_rays(origins, dirs, 50.0)

    r = make(d)
    r.set_build(2)                                            # the global build: scratch made at its first use
    got = r.render(wl.cameras, wl.fov, 1, **ALL)
    assert same(got, first)
    ng.inject_allocation_failure(0)
    with pytest.raises(ng.CudaError, match="out of memory"):
        r.set_instance_transforms(wl.matrices)
    ng.inject_allocation_failure(-1)
    assert same(r.render(wl.cameras, wl.fov, 1, **ALL), first)   # the previous tree is still in place
    _, failures = until_it_works(lambda: r.set_instance_transforms(wl.matrices))
    assert failures >= 1
    r.record_hits(True)                                       # the next render makes the hit-record arrays
    got, failures = until_it_works(lambda: r.render(wl.cameras, wl.fov, 1, **ALL))
    assert failures >= 1 and same(got, want)
    rays, failures = until_it_works(lambda: r.cast_rays(origins, dirs, 50.0))
    assert failures >= 1 and same(rays, want_rays)
    assert (want_rays["object_id"] > 0).mean() > 0.2
    del r, clean
    assert ng.device_bytes() == base


def test_failed_mesh_rebuild_can_be_made_again(torch_cuda):
    wl = scene()
    d = wl.desc
    mesh = d.meshes[0]
    v = mesh.vertices * np.float32([1.2, 0.9, 1.0])
    clean = make(d)
    clean.set_instance_transforms(wl.matrices)
    clean.update_mesh(0, v)
    want = clean.render(wl.cameras, wl.fov, 1, **ALL)
    r = make(d)
    r.set_instance_transforms(wl.matrices)
    _, failures = until_it_works(lambda: r.update_mesh(0, v))
    assert failures >= 1
    assert same(r.render(wl.cameras, wl.fov, 1, **ALL), want)
