"""Worlds across ranks (neraulgraphics_b200.sharding): the partition, and two gloo ranks on CPU that each
render their own worlds and gather every image, against one rank rendering them all. The per-rank renderer
here is the oracle, the CPU stand-in for each rank's GPU; the sharding logic is what is under test."""

import datetime
import os
import socket
import sys

import numpy as np
import pytest

from neraulgraphics_b200.sharding import row_range, world_range

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("worlds,size", [(5, 2), (4096, 8), (3, 4), (0, 2), (17, 1)])
def test_world_ranges_cover_every_world_once_in_order(worlds, size):
    ranges = [world_range(worlds, r, size) for r in range(size)]
    assert ranges[0][0] == 0 and ranges[-1][1] == worlds
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1 and sorted(sizes, reverse=True) == sizes
    with pytest.raises(ValueError):
        world_range(worlds, size, size)


@pytest.mark.parametrize("height,size", [(720, 8), (29, 2), (29, 8), (4, 1), (1, 1), (13, 3)])
def test_row_bands_are_whole_tiles_covering_every_row_once(height, size):
    bands = [row_range(height, r, size) for r in range(size)]
    assert bands[0][0] == 0 and bands[-1][0] + bands[-1][1] == height
    assert all(a[0] + a[1] == b[0] for a, b in zip(bands, bands[1:]))
    assert all(first % 4 == 0 and count >= 1 for first, count in bands)
    tiles = [(count + 3) // 4 for _, count in bands]
    assert max(tiles) - min(tiles) <= 1
    with pytest.raises(ValueError):
        row_range(height, 0, (height + 3) // 4 + 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, size, port, worlds, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import oracle as O
    from neraulgraphics_b200 import workloads
    from neraulgraphics_b200.scene import SceneDesc
    from neraulgraphics_b200.sharding import ShardedWorlds
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=120))
    try:
        wl = workloads.body_worlds(worlds=worlds, width=24, height=16, seed=3)
        d = wl.desc
        shard = ShardedWorlds(worlds)
        local = SceneDesc(d.width, d.height, shard.count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances)
        o = O.Oracle(local)
        o.bind_bodies(**wl.binding)
        o.set_body_poses(shard.take(wl.poses))
        img = o.render(shard.take(wl.cameras), wl.fov, 1, rgb=True, depth=True, object_ids=True)
        got = {k: shard.gather(torch.from_numpy(v)).numpy() for k, v in img.items()}
        slowest = shard.max_over_ranks(0.5 + rank)
        if rank == 0:
            full = O.Oracle(d)
            full.bind_bodies(**wl.binding)
            full.set_body_poses(wl.poses)
            want = full.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
            ok = all(np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)) for k in want)
            np.save(out, np.array([ok, slowest == size - 0.5, shard.start, shard.stop], dtype=np.float64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("worlds", [5, 2])
def test_two_ranks_render_their_worlds_and_gather_everything(tmp_path, worlds):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port, out = _free_port(), str(tmp_path / "rank0.npy")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, worlds, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ok, slowest, start, stop = np.load(out)
    assert ok and slowest and (start, stop) == (0, (worlds + 1) // 2)


def _ray_rank(rank, size, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import oracle as O
    import scenes
    from neraulgraphics_b200.sharding import ShardedRays
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=120))
    try:
        desc, mats, _ = scenes.scattered_boxes(1, 3000)
        el = np.radians(np.linspace(-15.0, 15.0, 16))
        az = np.radians(np.linspace(0.0, 360.0, 63, endpoint=False))
        e, a = np.meshgrid(el, az, indexing="ij")
        dirs = np.stack([np.cos(e) * np.sin(a), np.sin(e), -np.cos(e) * np.cos(a)], -1).reshape(1, -1, 3).astype(np.float32)
        dirs = dirs[:, :1001]  # an odd count: shares of 501 and 500
        origins = np.tile(np.float32([0.0, 0.0, -40.0]), (1, dirs.shape[1], 1))
        o = O.Oracle(desc)
        o.set_instance_transforms(mats)  # every rank: the whole scene, the same tree
        shard = ShardedRays(dirs.shape[1])
        hits = o.cast_rays(shard.take(origins), shard.take(dirs), 100.0)
        got = {k: shard.gather(torch.from_numpy(np.ascontiguousarray(v))).numpy() for k, v in hits.items()}
        if rank == 0:
            want = o.cast_rays(origins, dirs, 100.0)
            ok = all(np.array_equal(np.asarray(got[k]).view(np.uint8), np.asarray(want[k]).view(np.uint8)) for k in want)
            hit = float((want["object_id"] > 0).mean())
            np.save(out, np.array([ok, hit, shard.start, shard.stop], dtype=np.float64))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_one_worlds_rays():
    """One world's 1001 ray queries split over two gloo ranks (501 + 500), each holding the whole scene, then
    gathered in ray order: the same distances, normals and IDs as one rank casting them all."""
    import tempfile

    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as tmp:
        port, out = _free_port(), os.path.join(tmp, "rank0.npy")
        procs = [ctx.Process(target=_ray_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
        for p in procs:
            if p.is_alive():
                p.kill()
        assert all(p.exitcode == 0 for p in procs)
        ok, hit, start, stop = np.load(out)
    assert ok == 1.0 and hit > 0.2 and (start, stop) == (0, 501)


def _frame_rank(rank, size, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import oracle as O
    from neraulgraphics_b200 import workloads
    from neraulgraphics_b200.sharding import ShardedFrame
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=120))
    try:
        wl = workloads.icosphere_worlds(worlds=1, per_world=30, width=20, height=29, seed=11)
        shard = ShardedFrame(height=29)
        # Rank 0's matrices replicated to every rank: each builds the same tree.
        mats = torch.from_numpy(wl.matrices) if rank == 0 else torch.zeros(wl.matrices.shape, dtype=torch.float32)
        shard.broadcast(mats)
        o = O.Oracle(wl.desc)
        o.set_instance_transforms(mats.numpy())
        img = o.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
        band = {k: torch.from_numpy(np.ascontiguousarray(shard.take(v))) for k, v in img.items()}
        got = {k: shard.gather(v).numpy() for k, v in band.items()}
        slowest = shard.max_over_ranks(1.0 + rank)
        if rank == 0:
            full = O.Oracle(wl.desc)
            full.set_instance_transforms(wl.matrices)
            want = full.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
            ok = all(np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)) for k in want)
            hit = float((want["object_ids"] >= 34).mean())
            np.save(out, np.array([ok, hit, slowest, shard.first, shard.count], dtype=np.float64))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_one_pictures_rows():
    """One world's 29-row picture split over two gloo ranks (rows 0-15 and 16-28, whole 4-row tiles), the
    instance matrices broadcast from rank 0, the bands gathered in row order: the whole picture, bit for bit."""
    import tempfile

    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as tmp:
        port, out = _free_port(), os.path.join(tmp, "rank0.npy")
        procs = [ctx.Process(target=_frame_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
        for p in procs:
            if p.is_alive():
                p.kill()
        assert all(p.exitcode == 0 for p in procs)
        ok, hit, slowest, first, count = np.load(out)
    assert ok == 1.0 and hit > 0.1 and slowest == 2.0 and (first, count) == (0, 16)
