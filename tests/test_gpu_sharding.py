"""The sharding splits (neraulgraphics_b200.sharding) with the product's renderers: two ranks of a gloo process group,
each a process with its own BatchRenderer on cuda:0, render their share and gather it, against one renderer
doing all the work.

The ranks share one GPU here (every GPU call of this build has one). Nothing on the device waits for the other
rank: each rank's kernels touch only its own renderer, and the collectives (gloo) run on the host, so the two
processes are independent users of the GPU; on a node of several GPUs each rank takes its own with NCCL.

  - worlds: each rank its contiguous range of 9 worlds (5 + 4), the images gathered in world order;
  - rays: one world of 3,000 instances replicated, its 1,001 ray queries split 501 + 500;
  - rows: one picture's 29 rows split into bands of whole 4-row tiles (16 + 13), the instance matrices broadcast
    from rank 0, the bands gathered in row order.
Each gathered result must equal the single renderer's bit for bit.
"""

import datetime
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _same(got, want):
    return all(np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8), np.ascontiguousarray(want[k]).view(np.uint8))
               for k in want)


def _rank(kind, rank, size, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import sharding, workloads
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=120))
    try:
        ok, extra = False, 0.0
        if kind == "worlds":
            wl = workloads.body_worlds(worlds=9, width=40, height=24, seed=5)
            d = wl.desc
            shard = sharding.ShardedWorlds(9)
            r = ng.BatchRenderer(d.width, d.height, shard.count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                                 device="cuda:0")
            r.bind_bodies(**wl.binding)
            r.set_body_poses(shard.take(wl.poses))
            img = r.render(shard.take(wl.cameras), wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=2)
            got = {k: shard.gather(torch.from_numpy(np.ascontiguousarray(v))).numpy() for k, v in img.items()}
            extra = shard.max_over_ranks(1.0 + rank)
            if rank == 0:
                full = ng.BatchRenderer(d.width, d.height, 9, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                                        device="cuda:0")
                full.bind_bodies(**wl.binding)
                full.set_body_poses(wl.poses)
                ok = _same(got, full.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True, frame=2))
        elif kind == "rays":
            import scenes
            desc, mats, _ = scenes.scattered_boxes(1, 3000)
            el = np.radians(np.linspace(-15.0, 15.0, 16))
            az = np.radians(np.linspace(0.0, 360.0, 63, endpoint=False))
            e, a = np.meshgrid(el, az, indexing="ij")
            dirs = np.stack([np.cos(e) * np.sin(a), np.sin(e), -np.cos(e) * np.cos(a)], -1).reshape(1, -1, 3)[:, :1001]
            dirs = np.ascontiguousarray(dirs, np.float32)
            origins = np.tile(np.float32([0.0, 0.0, -40.0]), (1, dirs.shape[1], 1))
            r = ng.BatchRenderer(desc.width, desc.height, 1, 1, desc.spheres, desc.lights, desc.floor, desc.meshes,
                                 desc.instances, device="cuda:0")
            r.set_instance_transforms(mats)
            shard = sharding.ShardedRays(dirs.shape[1])
            hits = r.cast_rays(np.ascontiguousarray(shard.take(origins)), np.ascontiguousarray(shard.take(dirs)), 100.0)
            got = {k: shard.gather(torch.from_numpy(np.ascontiguousarray(v))).numpy() for k, v in hits.items()}
            if rank == 0:
                want = r.cast_rays(origins, dirs, 100.0)
                ok = _same(got, want)
                extra = float((want["object_id"] >= ng.OBJECT_INSTANCE).mean())
        else:
            wl = workloads.icosphere_worlds(worlds=1, per_world=30, width=20, height=29, seed=11)
            d = wl.desc
            shard = sharding.ShardedFrame(height=29)
            mats = torch.from_numpy(wl.matrices) if rank == 0 else torch.zeros(wl.matrices.shape, dtype=torch.float32)
            shard.broadcast(mats)
            r = ng.BatchRenderer(d.width, d.height, 1, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                                 device="cuda:0")
            r.set_instance_transforms(mats.numpy())
            shard.apply(r)
            band = r.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
            got = {k: shard.gather(torch.from_numpy(np.ascontiguousarray(v))).numpy() for k, v in band.items()}
            extra = float(shard.count)
            if rank == 0:
                full = ng.BatchRenderer(d.width, d.height, 1, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                                        device="cuda:0")
                full.set_instance_transforms(wl.matrices)
                ok = _same(got, full.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True))
        if rank == 0:
            np.save(out, np.array([ok, extra], dtype=np.float64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["worlds", "rays", "rows"])
def test_two_ranks_of_the_product_split_and_gather(torch_cuda, tmp_path, kind):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port, out = _free_port(), str(tmp_path / "rank0.npy")
    procs = [ctx.Process(target=_rank, args=(kind, r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ok, extra = np.load(out)
    assert ok == 1.0
    if kind == "worlds":
        assert extra == 2.0  # the slowest rank's figure, max over ranks
    elif kind == "rays":
        assert extra > 0.2
    else:
        assert extra == 16.0  # rank 0's band: rows 0-15
