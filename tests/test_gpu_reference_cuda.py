"""The product against the reference's own GPU path on the same seeded inputs, on the GPU.

The reference here is neraulgraphics 0.5.0's CUDA backend (src/cuda_backend.cu) and its instance-tree build
(src/cuda_tlas.cuh), compiled from its sources for sm_100 with its own flags by oracle/Makefile. Those flags
include -use_fast_math (CMakeLists.txt:127-131 in the reference), so its Morton keys divide by the world's
extent with the fast approximate division (cuda_tlas.cuh:99-115) and its shading uses fast sines, powers and
square roots: bit-exactness with the IEEE path (the reference's CPU backend, which the oracle and the product
follow) is not possible, and the test reports and bounds the differences instead:
  - Morton keys that differ and sorted positions holding a different instance (same matrices into both builds);
    and, since both sorts are stable radix sorts, worlds whose keys all agree must agree on their sorted order;
  - pixels whose object ID differs, pixels of the same object whose depth differs by more than 1e-5 relative,
    and pixels whose RGB differs by more than one level.
Bounds: object IDs as the reference bounds two valid trees of one scene (1 pixel in 2000,
tests/test_batch.cpp:335-374 there), depth beyond 1e-5 relative in at most 1 pixel in 1000 of those, RGB beyond
one level in at most 1 pixel in 200.
"""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu

needs_ref_cuda = pytest.mark.skipif(not (O.reference_available(cuda=True) and O.ref_tlas_available()),
                                    reason="the reference's CUDA backend is not built (make -C oracle ref-cuda)")


def product(d):
    return ng.BatchRenderer(d.width, d.height, d.world_count, d.cameras_per_world, d.spheres, d.lights, d.floor,
                            d.meshes, d.instances, device="cuda:0")


def tree_differences(desc, ours, matrices):
    """Counts of differing keys and sorted positions against the reference's GPU build of the same matrices."""
    W, P = desc.world_count, desc.per_world
    bounds = O.Oracle(desc).blas()["bounds"][[inst.mesh for inst in desc.instances]]
    ref = O.ref_tlas_cuda(W, P, bounds, matrices)
    key_diff = ours["keys"] != ref["keys"]
    pos_diff = ours["sorted_ids"] != ref["sorted_ids"]
    same_keys = ~key_diff.reshape(W, P).any(1)
    # A world whose keys all agree is sorted alike by both stable sorts.
    assert not (pos_diff.reshape(W, P) & same_keys[:, None]).any()
    if same_keys.all():  # the same keys make the same tree, node for node
        assert np.array_equal(ours["nodes"][:, [3, 7]], ref["nodes"][:, [3, 7]])
        assert np.array_equal(ours["roots"], ref["roots"])
    return int(key_diff.sum()), int(pos_diff.sum()), int((~same_keys).sum())


def image_differences(got, ref):
    ids = got["object_ids"] != ref["object_ids"]
    same = ~ids & np.isfinite(got["depth"]) & np.isfinite(ref["depth"])
    rel = np.abs(got["depth"] - ref["depth"]) / np.maximum(np.abs(ref["depth"]), 1e-30)
    depth = same & (rel > 1e-5)
    rgb = np.abs(got["rgb"].astype(int) - ref["rgb"].astype(int)).max(-1) > 1
    return ids.size, int(ids.sum()), int(depth.sum()), int(rgb.sum())


def check_bounds(label, counts, keys):
    n, ids, depth, rgb = counts
    k, pos, worlds = keys
    print(f"\n{label}: keys differing {k}, sorted positions differing {pos} (in {worlds} worlds); "
          f"pixels {n}: object ID {ids} ({ids / n:.2e}), depth > 1e-5 rel {depth} ({depth / n:.2e}), "
          f"RGB > 1 level {rgb} ({rgb / n:.2e})")
    assert ids <= n / 2000
    assert depth <= n / 1000
    assert rgb <= n / 200


@needs_ref_cuda
def test_icosphere_worlds_against_the_references_cuda_backend(torch_cuda):
    """16 worlds' scene (8 icospheres of 320 triangles over a floor) at 256 worlds, placed by matrices."""
    wl = workloads.icosphere_worlds(worlds=256, seed=1)
    d = wl.desc
    r, ref = product(d), O.Reference(d, cuda=True)
    r.set_instance_transforms(wl.matrices)
    ref.set_instance_transforms(wl.matrices)
    got = r.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    want = ref.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    keys = tree_differences(d, r.inspect_tlas(), wl.matrices)
    check_bounds("icosphere worlds 256 x 64x64", image_differences(got, want), keys)


@needs_ref_cuda
def test_body_worlds_against_the_references_cuda_backend(torch_cuda):
    """4096 worlds x 20 bodies of three meshes at 64x64, moved by the random walk: each side composes the body
    poses itself (the reference with its fast-math quaternion arithmetic), builds and renders."""
    wl = workloads.body_worlds(seed=2)
    d = wl.desc
    poses = workloads.random_walk(wl.poses, 2, seed=5)[-1]
    r, ref = product(d), O.Reference(d, cuda=True)
    for x in (r, ref):
        x.bind_bodies(**wl.binding)
        x.set_body_poses(poses)
    got = r.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    want = ref.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    ours = r.inspect_tlas()
    keys = tree_differences(d, ours, ours["matrices"])
    check_bounds("body worlds 4096 x 64x64", image_differences(got, want), keys)
