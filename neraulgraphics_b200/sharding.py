"""Worlds across GPUs: one process per GPU, each rendering its own contiguous range of the worlds.

Worlds are independent, so the render shards with no exchange on the data path: every rank composes, builds
and renders its own worlds, and its images stay on its GPU for the consumer there (a policy, a loss). A
consumer that wants every image calls gather(), one all-gather over the process group (NCCL over NVLink on
GPUs; gloo on CPUs). Timing is the slowest rank's: max_over_ranks().

    import torch.distributed as dist
    dist.init_process_group("nccl")
    shard = ShardedWorlds(world_count=16384)              # this rank's worlds: shard.start .. shard.stop
    r = BatchRenderer(64, 64, shard.count, ...)           # a renderer of those worlds only
    r.set_body_poses(shard.take(all_poses))               # or poses made on this rank for its worlds
    images = r.render(shard.take(all_cameras), zero_copy=True)
    everything = shard.gather(images["depth"])            # (16384, 64, 64) on every rank, if wanted
"""

from __future__ import annotations


def world_range(world_count: int, rank: int, world_size: int) -> tuple[int, int]:
    """[start, stop) of rank's worlds: contiguous ranges, in rank order, whose sizes differ by at most one."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} is not in a group of {world_size}")
    if world_count < 0:
        raise ValueError(f"world_count must be 0 or more, got {world_count}")
    base, extra = divmod(world_count, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def row_range(height: int, rank: int, world_size: int, tile: int = 4) -> tuple[int, int]:
    """(first, count) of rank's rows of an image height rows tall: contiguous bands of whole tiles of `tile`
    rows (the render kernels' tile height), in rank order, whose tile counts differ by at most one; the last
    band ends at the image's last row. Every rank gets at least one row."""
    if height < 1:
        raise ValueError(f"height must be 1 or more, got {height}")
    tiles = (height + tile - 1) // tile
    if tiles < world_size:
        raise ValueError(f"{world_size} ranks cannot share {tiles} tiles of {tile} rows ({height} rows)")
    start, stop = world_range(tiles, rank, world_size)
    first = start * tile
    return first, min(stop * tile, height) - first


class _Group:
    """The process group's rank and size (one rank when torch.distributed is not initialised), and the
    collectives every split uses."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.size = 0, 1

    def broadcast(self, tensor, src: int = 0):
        """tensor as rank src holds it, on every rank, in place (the scene's inputs replicated from one rank:
        every rank then builds the same tree). Returns tensor."""
        import torch.distributed as dist
        if self.size > 1:
            dist.broadcast(tensor, src, group=self.group)
        return tensor

    def max_over_ranks(self, value: float, device=None) -> float:
        """The largest value over the ranks (a time: the job takes as long as its slowest rank)."""
        import torch
        import torch.distributed as dist
        if self.size == 1:
            return float(value)
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return float(t.item())


class ShardedWorlds(_Group):
    """This rank's share of world_count worlds in a torch.distributed process group (the default group when
    group is None; one rank when torch.distributed is not initialised)."""

    def __init__(self, world_count: int, group=None):
        super().__init__(group)
        self.world_count = world_count
        self.start, self.stop = world_range(world_count, self.rank, self.size)
        self.ranges = [world_range(world_count, r, self.size) for r in range(self.size)]

    @property
    def count(self) -> int:
        return self.stop - self.start

    def take(self, per_world):
        """This rank's slice of an array or tensor whose first axis runs over every world."""
        if len(per_world) != self.world_count:
            raise ValueError(f"expected {self.world_count} worlds on the first axis, got {len(per_world)}")
        return per_world[self.start:self.stop]

    def gather(self, local):
        """Every rank's local tensor (first axis: its worlds, or its views world-major with a fixed number per
        world) concatenated in world order, on every rank: one all-gather of equal-sized, padded pieces."""
        import torch
        import torch.distributed as dist
        if self.size == 1:
            return local
        # Every rank's row count; the ranks must agree on the rows per world, and the largest piece sets the
        # padded size of the all-gather.
        rows = torch.tensor([local.shape[0], self.count], dtype=torch.int64, device=local.device)
        all_rows = [torch.zeros_like(rows) for _ in range(self.size)]
        dist.all_gather(all_rows, rows, group=self.group)
        per_world = {int(r[0]) / int(r[1]) for r in all_rows if int(r[1]) > 0}
        if len(per_world) > 1 or any(float(p) != int(p) for p in per_world):
            raise ValueError("every rank's local tensor must hold the same number of rows per world")
        pad = max(int(r[0]) for r in all_rows)
        piece = torch.zeros((pad,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
        piece[:local.shape[0]] = local
        pieces = [torch.empty_like(piece) for _ in range(self.size)]
        dist.all_gather(pieces, piece, group=self.group)
        return torch.cat([p[:int(r[0])] for p, r in zip(pieces, all_rows)], 0)


class ShardedRays(_Group):
    """This rank's share of every world's rays: for one large world (or a few) whose ray queries outnumber its
    worlds, such as a LiDAR sweep of one scene. Every rank holds the whole scene (the same instance matrices,
    so the same tree) and casts a contiguous range of each world's rays; gather() puts the results back in
    ray order. The ray queries are independent, so nothing is exchanged until the gather.

        shard = ShardedRays(rays_per_world=131072)
        hits = r.cast_rays(shard.take(origins), shard.take(directions), max_distance)
        everything = {k: shard.gather(v) for k, v in hits.items()}      # (worlds, 131072, ...) on every rank
    """

    def __init__(self, rays_per_world: int, group=None):
        super().__init__(group)
        self.rays_per_world = rays_per_world
        self.start, self.stop = world_range(rays_per_world, self.rank, self.size)
        self.ranges = [world_range(rays_per_world, r, self.size) for r in range(self.size)]

    @property
    def count(self) -> int:
        return self.stop - self.start

    def take(self, per_ray):
        """This rank's rays of an array or tensor shaped (worlds, rays_per_world, ...)."""
        if per_ray.shape[1] != self.rays_per_world:
            raise ValueError(f"expected {self.rays_per_world} rays per world on the second axis, got {per_ray.shape[1]}")
        return per_ray[:, self.start:self.stop]

    def gather(self, local):
        """Every rank's (worlds, its rays, ...) tensor joined along the rays in ray order, on every rank: one
        all-gather of pieces padded to the largest share."""
        import torch
        import torch.distributed as dist
        if self.size == 1:
            return local
        pad = max(b - a for a, b in self.ranges)
        piece = torch.zeros((local.shape[0], pad) + tuple(local.shape[2:]), dtype=local.dtype, device=local.device)
        piece[:, :local.shape[1]] = local
        pieces = [torch.empty_like(piece) for _ in range(self.size)]
        dist.all_gather(pieces, piece, group=self.group)
        return torch.cat([p[:, :b - a] for p, (a, b) in zip(pieces, self.ranges)], 1)


class ShardedFrame(_Group):
    """This rank's band of rows of every view's image: for one large picture (or a few) split across GPUs.
    Every rank holds the whole scene (the same instance matrices, so the same tree; broadcast() replicates
    them from one rank) and renders rows [first, first + count) of each view (BatchRenderer.set_rows), with
    the whole image's rays and random streams, so the joined bands are the whole image's pixels exactly.
    Bands are whole tiles of 4 rows; nothing is exchanged until the gather.

        shard = ShardedFrame(height=720)
        shard.apply(r)                                                   # r.set_rows(shard.first, shard.count)
        images = r.render(cams, zero_copy=True, rgb=True, depth=True)    # (views, shard.count, 1280, ...)
        everything = {k: shard.gather(v) for k, v in images.items()}     # (views, 720, 1280, ...) on every rank
    """

    def __init__(self, height: int, group=None):
        super().__init__(group)
        self.height = height
        self.ranges = [row_range(height, r, self.size) for r in range(self.size)]
        self.first, self.count = self.ranges[self.rank]

    def apply(self, renderer) -> None:
        """Sets renderer to draw this rank's rows."""
        if renderer.height != self.height:
            raise ValueError(f"the renderer's images are {renderer.height} rows tall, the frame {self.height}")
        renderer.set_rows(self.first, self.count)

    def take(self, per_pixel):
        """This rank's rows of an array or tensor shaped (views, height, ...)."""
        if per_pixel.shape[1] != self.height:
            raise ValueError(f"expected {self.height} rows on the second axis, got {per_pixel.shape[1]}")
        return per_pixel[:, self.first:self.first + self.count]

    def gather(self, local):
        """Every rank's (views, its rows, ...) tensor joined along the rows in image order, on every rank: one
        all-gather of pieces padded to the largest band."""
        import torch
        import torch.distributed as dist
        if local.shape[1] != self.count:
            raise ValueError(f"expected this rank's {self.count} rows on the second axis, got {local.shape[1]}")
        if self.size == 1:
            return local
        pad = max(c for _, c in self.ranges)
        piece = torch.zeros((local.shape[0], pad) + tuple(local.shape[2:]), dtype=local.dtype, device=local.device)
        piece[:, :local.shape[1]] = local
        pieces = [torch.empty_like(piece) for _ in range(self.size)]
        dist.all_gather(pieces, piece, group=self.group)
        return torch.cat([p[:, :c] for p, (_, c) in zip(pieces, self.ranges)], 1)
