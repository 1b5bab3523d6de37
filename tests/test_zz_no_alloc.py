"""The tree build that allocates nothing (ngb_build_tlas_noalloc), against the renderer's own build.

This entry point serves callers that cannot call cudaMalloc, such as a framework that owns the GPU's memory
through its own pool, so its scratch lives in a static device array instead. Here the test allocates the inputs and outputs (with PyTorch) and checks that two calls in a row
give exactly the trees ngb_set_instance_transforms builds for the same matrices, and that the caller's error
word reads 0 after each (a build whose box climb overran would set it). It sorts last, so a run that
stops at its first failure has run every other test first, and it passes alone in a fresh process as well.
"""

import ctypes as C

import numpy as np
import pytest

import neraulgraphics_b200 as ng
from neraulgraphics_b200 import workloads
from neraulgraphics_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def test_static_scratch_build_matches_the_renderers_build_twice(torch_cuda):
    torch = torch_cuda
    wl = workloads.body_worlds(worlds=300, seed=4)
    d = wl.desc
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device="cuda:0")
    r.bind_bodies(**wl.binding)
    built = ng.build_meshes(d.meshes)
    slot_mesh = [inst.mesh for inst in d.instances]
    bounds = torch.from_numpy(np.ascontiguousarray(built["bounds"][slot_mesh])).cuda()
    blas_root = torch.from_numpy(np.ascontiguousarray(built["roots"][slot_mesh], dtype=np.int32)).cuda()
    W, P = d.world_count, d.per_world
    n = W * P
    records = torch.empty((n, 16), dtype=torch.float32, device="cuda:0")
    keys = torch.empty(n, dtype=torch.int64, device="cuda:0")
    ids = torch.empty(n, dtype=torch.int32, device="cuda:0")
    nodes = torch.empty((2 * n - 1, 8), dtype=torch.int32, device="cuda:0")
    roots = torch.empty(W, dtype=torch.int32, device="cuda:0")
    error = torch.full((1,), -7, dtype=torch.int32, device="cuda:0")
    L = lib()
    stream = torch.cuda.current_stream().cuda_stream
    for step in workloads.random_walk(wl.poses, 2, seed=9):
        r.set_body_poses(step)
        want = r.inspect_tlas()
        mats = torch.from_numpy(want["matrices"]).cuda()
        for t in (records, keys, ids, nodes, roots):
            t.fill_(-7)  # anything the call leaves unwritten shows up
        ptr = lambda t: C.c_void_p(t.data_ptr())
        check(L.ngb_build_tlas_noalloc(W, P, ptr(mats), ptr(bounds), ptr(blas_root), ptr(records), ptr(keys),
                                       ptr(ids), ptr(nodes), ptr(roots), ptr(error), C.c_void_p(stream)))
        torch.cuda.synchronize()
        assert int(error.item()) == 0
        got_nodes = nodes.cpu().numpy()
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), want["keys"])
        assert np.array_equal(ids.cpu().numpy(), want["sorted_ids"])
        assert np.array_equal(roots.cpu().numpy(), want["roots"])
        assert np.array_equal(got_nodes[:, [3, 7]], want["nodes"][:, [3, 7]])
        assert np.array_equal(got_nodes[:, [0, 1, 2, 4, 5, 6]].view(np.float32),
                              want["nodes"][:, [0, 1, 2, 4, 5, 6]].view(np.float32))
        rec = records.cpu().numpy()
        assert np.array_equal(rec[:, 12].view(np.int32), built["roots"][slot_mesh * W])
        assert np.array_equal(rec[:, 13].view(np.int32), np.tile(np.arange(P, dtype=np.int32), W))


def test_static_scratch_build_rejects_sizes_beyond_its_limit(torch_cuda):
    L = lib()
    nul = C.c_void_p(16)
    status = L.ngb_build_tlas_noalloc(70, 1000, nul, nul, nul, nul, nul, nul, nul, nul, None, None)
    assert status == 1
    assert "at most 65536" in L.ngb_last_error(None).decode()
