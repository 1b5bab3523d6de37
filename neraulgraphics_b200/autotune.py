"""Picks the render kernel's launch shape for a workload by timing it.

For worlds of at most 256 instances the tile kernel runs, and its shape is the CTA size, the register budget
per thread (which sets how many warps an SM holds), the rays a warp takes per fetch of work (tiles of 32 rays:
1, 2 or 4) and the camera tile's shape (a pixel's picture and centre rays paired on a 4 x 4 tile, or 8 x 4 tiles
of one kind of ray in two passes). Otherwise the persistent kernel runs, and its
shape adds the refill threshold (how many of a warp's lanes must be free before it takes new pixels) and the
leaf batch. The best depends on the scene (how long rays walk, how much they vary), so it is measured on the
caller's own renderer and cameras, with CUDA events, and remembered in a JSON cache keyed by the GPU and the
workload's shape.

    from neraulgraphics_b200.autotune import tune
    best = tune(renderer, cameras, fov=1.0, rgb=True, depth=True, object_ids=True)
"""

from __future__ import annotations

import json
import os
import time

CANDIDATES = [(threads, regs, refill, batch) for threads, regs in ((128, 64), (256, 64), (128, 48), (64, 64))
              for refill in (16, 24, 28) for batch in (1, 8, 16, 24)]
TILE_CANDIDATES = [(128, 48, 0, 0), (128, 56, 0, 0), (128, 64, 0, 0), (256, 64, 0, 0)]
TILE_FETCH = (1, 2, 4)       # tiles of 32 rays a warp takes per fetch
TILE_PAIRED = (True, False)  # a pixel's two camera rays on one 4 x 4 tile, or 8 x 4 tiles of one kind
TILE_MAX_INSTANCES = 256


def cache_path() -> str:
    return os.environ.get("NGB_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "neraulgraphics_b200", "tuning.json"))


def _key(renderer, outputs) -> str:
    import torch
    name = torch.cuda.get_device_name(renderer._device)
    return (f"{name}|{renderer.world_count}x{renderer.cameras_per_world}|{renderer.width}x{renderer.rows[1]}|"
            f"{renderer.instances_per_world}|{outputs}")


def _apply(renderer, shape: dict) -> None:
    if shape["kernel"] == 3:
        renderer.set_tuning(kernel=3, threads_per_block=shape["threads"], registers=shape["registers"])
        renderer.set_tile_shape(shape.get("fetch", 1), shape.get("paired", True))
    else:
        renderer.set_tuning(kernel=shape["kernel"], threads_per_block=shape["threads"], refill_lanes=shape["refill"],
                            registers=shape["registers"], leaf_batch=shape["leaf_batch"])


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def tune(renderer, cameras, fov=1.0, *, rgb=True, depth=False, normals=False, object_ids=False, repeats=3,
         use_cache=True, budget_s=60.0) -> dict:
    """Times every candidate shape on this renderer and these cameras (device tensors), sets the fastest and
    returns {"kernel", "threads", "registers", "refill", "leaf_batch", "fetch", "paired", "ms", "timings"}."""
    import torch
    outputs = dict(rgb=rgb, depth=depth, normals=normals, object_ids=object_ids)
    # Worlds of at most TILE_MAX_INSTANCES instances: the tile kernels' shapes. Larger worlds: the persistent
    # kernel's shapes and the tile kernels walking each world's tree as a packet, whichever is faster here.
    kernel = 3 if renderer.instances_per_world <= TILE_MAX_INSTANCES else 2
    candidates = ([(3,) + c + (f, p) for c in TILE_CANDIDATES for f in TILE_FETCH for p in TILE_PAIRED]
                  if kernel == 3 else
                  [(2,) + c + (1, True) for c in CANDIDATES] +
                  [(3,) + c + (1, True) for c in TILE_CANDIDATES + [(128, 80, 0, 0)]])
    key = _key(renderer, tuple(sorted(k for k, v in outputs.items() if v))) + f"|kernel{kernel}"
    cache = _load() if use_cache else {}
    if key in cache:
        best = cache[key]
        _apply(renderer, best)
        return dict(best, cached=True)
    timings = []
    start = time.perf_counter()
    for kind, threads, regs, refill, batch, fetch, paired in candidates:
        shape = {"kernel": kind, "threads": threads, "refill": refill, "registers": regs, "leaf_batch": batch,
                 "fetch": fetch, "paired": paired}
        _apply(renderer, shape)
        renderer.render(cameras, fov, 1, zero_copy=True, **outputs)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            renderer.render(cameras, fov, 1, zero_copy=True, **outputs)
        e1.record()
        e1.synchronize()
        timings.append(dict(shape, ms=e0.elapsed_time(e1) / repeats))
        if time.perf_counter() - start > budget_s:
            break
    best = min(timings, key=lambda t: t["ms"])
    _apply(renderer, best)
    result = dict(best, timings=timings)
    if use_cache:
        cache[key] = {k: best[k] for k in ("kernel", "threads", "registers", "refill", "leaf_batch", "fetch", "paired",
                                           "ms")}
        try:
            os.makedirs(os.path.dirname(cache_path()), exist_ok=True)
            with open(cache_path(), "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    return result
