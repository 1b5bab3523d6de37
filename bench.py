#!/usr/bin/env python
"""Benchmark of the batched sensor-rendering path: images/s at 4096 worlds x 64x64, RGB + depth + object ID.

One step = one simulation step of the workload: every body of every world moves (a seeded Gaussian random
walk), the instance matrices are composed and every world's tree is rebuilt (set_body_poses), then every
view is rendered (render). Scenes are seeded synthetic stand-ins for recorded simulator poses
(neraulgraphics_b200.workloads.body_worlds).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one rank per GPU: each rank renders its own 4096 worlds (weak scaling, no
collective on the data path); the time is the max over ranks.

value: device-resident inputs (poses and cameras already on the GPU), CUDA events per step, L2 flushed
between steps. e2e: the public API with host buffers: pinned host poses in, images copied back to pinned
host memory, every step. --impl reference times the reference's own CPU backend (compiled from its sources
into oracle/_ref/) on a bounded sample of worlds per step, with every host core, and reports beside it the
reference's CUDA backend (built the same way) on the whole workload on the GPU ("reference_cuda").
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "images/s at 4096x64x64 RGB+depth+ID (body poses -> LBVH rebuild -> render, per step)"
UNIT = "images/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--worlds", type=int, default=4096)
    p.add_argument("--e2e-steps", type=int, default=100)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-reference-cuda", action="store_true",
                   help="--impl reference: skip timing the reference's CUDA backend on the GPU")
    p.add_argument("--no-autotune", action="store_true", help="use the library's default kernel shape")
    p.add_argument("--config", default="body_worlds",
                   choices=["body_worlds", "large_world", "differentiable", "uneven", "mesh_update"],
                   help="body_worlds: the headline (4096 worlds x 64x64); large_world: one world of 100,000 "
                        "instances at 1280x720 with a 64 x 2048 LiDAR sweep, poses redrawn every frame; "
                        "differentiable: 1024 worlds x 128x128 depth+normals, forward+backward against forward; "
                        "uneven: 2048 worlds of 1..200 instances at 32/64/128 px, one CUDA graph per step, against "
                        "bucketed plain renderers")
    p.add_argument("--no-forms", action="store_true",
                   help="body_worlds: leave out the differentiable and uneven sub-objects of the line")
    p.add_argument("--profile", action="store_true",
                   help="device-resident steps only (no autotune, e2e, CPU or reference arms): for ncu captures")
    return p.parse_args()


def workload_config(worlds, extra=None):
    cfg = {"workload": f"body_worlds: {worlds} worlds x 20 bodies (icosphere 1280 / box 12 / cylinder 512 tris), "
                       f"64x64, 1 light (soft shadows), spp 1, RGB+depth+ID, random-walk poses every step",
           "worlds_per_gpu": worlds, "width": 64, "height": 64, "instances_per_world": 20}
    cfg.update(extra or {})
    return cfg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 50 ms while running. Entering waits (up to 5 s) for
    nvidia-smi's first sample, so that its start-up (NVML initialisation, which can hold up this process's launches
    for milliseconds) ends before the timed region begins; the summary counts only the samples taken after that,
    or the last earlier one when the region was shorter than one sampling period."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.start = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        end = time.monotonic() + 5.0
        while self.proc and not self.lines and self.proc.poll() is None and time.monotonic() < end:
            time.sleep(0.01)
        self.start = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.start:] or self.lines[-1:]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


PROFILE = os.path.join(ROOT, "profiles", "camera_tiles_kernel_body_worlds.md")


def traffic_per_image():
    """DRAM bytes per image of the camera kernel, from the committed ncu summary (or None)."""
    try:
        for line in open(PROFILE):
            if line.startswith("dram_bytes_per_image:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def issue_figures():
    """The camera kernel's issue-side counters from the committed ncu summary's full capture: issue active (% of
    peak) and threads per warp instruction (of 32), or None."""
    want = {"issue active (% of peak)": "issue_active_pct", "threads per warp instruction": "threads_per_warp_instruction",
            "warps active (% of peak)": "warps_active_pct"}
    out = {}
    try:
        for line in open(PROFILE):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) >= 2 and cells[0] in want:
                out[want[cells[0]]] = float(cells[1])
    except (OSError, ValueError):
        return None
    if not out:
        return None
    out["source"] = "profiles/camera_tiles_kernel_body_worlds.md (ncu --set full, 1024 worlds)"
    return out


def algorithmic_bytes_per_image(wl, blas_bytes):
    """Compulsory bytes of one image of the body-worlds step, each counted once: the outputs (RGB 3, depth 4 and
    object ID 4 bytes per pixel); the inputs (the camera's 48 bytes and the world's body poses, 28 per body); and
    the tree build: per instance its matrix written and read (48 + 48), its inverse written (48), its box written
    and read (24 + 24) and its key and id through a two-pass sort (16 bytes, 2 reads and 2 writes); per world its
    2P - 1 nodes written (32 each); and the shared meshes' nodes and triangles read once per step, spread over the
    step's images."""
    d = wl.desc
    P = d.per_world
    out = d.height * d.width * (3 + 4 + 4)
    inputs = 48 + wl.binding["bodies_per_world"] * 28
    build = P * (48 + 48 + 48 + 24 * 2 + 16 * 4) + (2 * P - 1) * 32 + blas_bytes / d.view_count
    return out + inputs + build


def l2_copy_gbs(torch, dev, mib=32, copies=50, replays=10):
    """Copy bandwidth between two buffers that stay in L2 (2 x 32 MiB), read + write bytes over CUDA-event time, the
    copies captured in a CUDA graph so that launches do not separate them: this GPU's on-chip figure for byte rates
    served from cache (9.75 TB/s measured on a B200, against 6.44 TB/s for a copy through HBM)."""
    a = torch.ones(mib << 18, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(copies):
            b.copy_(a)
    graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(replays):
        graph.replay()
    e1.record()
    e1.synchronize()
    gbs = 2 * a.numel() * 4 * copies * replays / (e0.elapsed_time(e1) / 1000.0) / 1e9
    del graph
    return gbs


def cpu_baseline(wl, steps_poses, seconds, sample_worlds=64, count_worlds=16):
    """The reference's own CPU backend (oracle/_ref/libngref.so) on the first sample_worlds worlds of the
    workload, every host core: images/s. The CPU leg also renders the first count_worlds worlds with the
    instrumented port (oracle/), which counts the rays the path traces per image (a centre ray and a picture
    ray per pixel, a shadow ray per lit picture hit) and the bytes their walks fetch (32 per node, 64 per
    child-box pair, 48 per instance inverse, 48 per triangle): returned beside the timing as "counts"."""
    import oracle as O
    from neraulgraphics_b200.scene import SceneDesc
    d = wl.desc
    desc = SceneDesc(d.width, d.height, count_worlds, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances)
    o = O.Oracle(desc)
    o.bind_bodies(**wl.binding)
    o.set_body_poses(wl.poses[:count_worlds])
    o.render(wl.cameras[:count_worlds], wl.fov, 1, rgb=True, depth=True, object_ids=True)
    walked, rays = o.traversal_bytes()
    counts = {"rays_per_image": rays / count_worlds, "traversal_bytes_per_image": walked / count_worlds,
              "sample": f"the first {count_worlds} worlds, step 0 poses"}
    if not O.reference_available():
        return {"unavailable": "oracle/_ref was not built", "counts": counts}
    desc = SceneDesc(d.width, d.height, sample_worlds, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances)
    cores = os.cpu_count() or 1
    ref = O.Reference(desc, threads=cores)
    ref.bind_bodies(**wl.binding)
    cams = wl.cameras[:sample_worlds]
    ref.set_body_poses(steps_poses[0][:sample_worlds])
    ref.render(cams, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    n, t0 = 0, time.perf_counter()
    while True:
        ref.set_body_poses(steps_poses[(n + 1) % len(steps_poses)][:sample_worlds])
        ref.render(cams, wl.fov, 1, rgb=True, depth=True, object_ids=True)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 200:
            break
    return {"value": sample_worlds * n / el, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{n} steps of {sample_worlds} of the {d.world_count} worlds (set_body_poses + render_host, "
                      f"RGB+depth+ID), NERAULGRAPHICS_THREADS={cores}, {el:.1f} s", "counts": counts}


def reference_cuda(wl, torch, poses_dev, cams_dev, steps, warmup):
    """The reference's own CUDA backend (src/cuda_backend.cu built for sm_100 with its flags) on the same
    workload and the same device-resident inputs: images/s, CUDA events on its (legacy default) stream."""
    import oracle as O
    if not O.reference_available(cuda=True):
        return None
    ref = O.Reference(wl.desc, cuda=True)
    ref.bind_bodies(**wl.binding)
    outputs = 1 | 2 | 8
    for s in range(warmup):
        ref.set_body_poses(poses_dev[s].data_ptr(), device=True)
        ref.render_device(cams_dev.data_ptr(), wl.fov, 1, outputs)
    torch.cuda.synchronize()
    stream = torch.cuda.default_stream()
    times = []
    for s in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ref.set_body_poses(poses_dev[warmup + s].data_ptr(), device=True)
        ref.render_device(cams_dev.data_ptr(), wl.fov, 1, outputs)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    return {"value": wl.desc.view_count / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
            "kernel_ms_render": ref.last_kernel_ms,
            "what": "neraulgraphics 0.5.0 CudaBackend (set_body_poses + render_batch, RGB+depth+ID), sm_100, "
                    "-use_fast_math, same inputs on the device, median step"}


def run_ours(args, rank, world, local_rank, dist):
    import torch

    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import workloads

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    K, W = args.steps, args.warmup
    wl = workloads.body_worlds(worlds=args.worlds, seed=rank)
    steps_np = workloads.random_walk(wl.poses, W + K, seed=1 + rank)
    d = wl.desc
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device=dev)
    r.bind_bodies(**wl.binding)
    poses_dev = torch.from_numpy(steps_np).to(dev)
    cams_dev = torch.from_numpy(wl.cameras).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    kw = dict(rgb=True, depth=True, object_ids=True, zero_copy=True)
    tuned = None
    r.set_body_poses(poses_dev[0])
    if not args.no_autotune and not args.profile:
        from neraulgraphics_b200.autotune import tune
        tuned = tune(r, cams_dev, wl.fov, rgb=True, depth=True, object_ids=True, use_cache=False)
        for t in sorted(tuned["timings"], key=lambda t: t["ms"])[:12]:
            print("autotune", t, file=sys.stderr)
    for s in range(W):
        r.set_body_poses(poses_dev[s])
        r.render(cams_dev, wl.fov, 1, **kw)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with ClockSampler(local_rank) as clocks:
        for s in range(K):
            flush.zero_()
            e0, e1, e2 = ev[s]
            e0.record()
            r.set_body_poses(poses_dev[W + s])
            e1.record()
            r.render(cams_dev, wl.fov, 1, **kw)
            e2.record()
        torch.cuda.synchronize()
    build_ms = [a.elapsed_time(b) for a, b, _ in ev]
    render_ms = [b.elapsed_time(c) for _, b, c in ev]
    total_ms = sum(build_ms) + sum(render_ms)
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    views = d.view_count
    value = world * views * K / (total_ms / 1000.0)
    # Per-kernel GPU times of the render, from the library's events between its launches (untimed renders).
    stage = []
    for s in range(5):
        r.render(cams_dev, wl.fov, 1, **kw)
        stage.append(r.last_stage_ms)
    stage_ms = [statistics.median(x[i] for x in stage) for i in range(len(stage[0]))]
    if args.profile:
        if rank == 0:
            return {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K,
                    "warmup": W, "ms_per_step": round(total_ms / K, 4), "profile_run": True,
                    "stage_ms": [round(x, 4) for x in stage_ms]}
        return None

    # End to end through the public API with host buffers: every step, that step's poses and cameras go from
    # pinned host memory to the GPU (on an upload stream, while the step before renders), the renderer builds
    # and renders into one of two device image sets, and the images come back to pinned host memory on a copy
    # stream while the next step renders.
    pinned_poses = torch.from_numpy(steps_np).pin_memory()
    pinned_cams = torch.from_numpy(wl.cameras).pin_memory()
    shapes = {"rgb": ((views, 64, 64, 3), torch.uint8), "depth": ((views, 64, 64), torch.float32),
              "object_ids": ((views, 64, 64), torch.int32)}
    dev_out = [{k: torch.empty(sh, dtype=dt, device=dev) for k, (sh, dt) in shapes.items()} for _ in range(2)]
    host_out = [{k: torch.empty(sh, dtype=dt).pin_memory() for k, (sh, dt) in shapes.items()} for _ in range(2)]
    dev_poses = [torch.empty_like(pinned_poses[0], device=dev) for _ in range(2)]
    dev_cams = [torch.empty_like(pinned_cams, device=dev) for _ in range(2)]
    copier, uploader = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    rendered = [torch.cuda.Event() for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    uploaded = [torch.cuda.Event() for _ in range(2)]
    ekw = dict(rgb=True, depth=True, object_ids=True)
    KE = max(1, args.e2e_steps)

    def upload(s):
        i = s % 2
        uploader.wait_event(rendered[i])  # the render two steps back has read this input set
        with torch.cuda.stream(uploader):
            dev_poses[i].copy_(pinned_poses[W + s % K], non_blocking=True)
            dev_cams[i].copy_(pinned_cams, non_blocking=True)
            uploaded[i].record()

    def e2e_steps(n):
        upload(0)
        for s in range(n):
            i = s % 2
            cur = torch.cuda.current_stream()
            cur.wait_event(copied[i])    # the copy out of this image set has finished
            cur.wait_event(uploaded[i])  # this step's poses and cameras are on the device
            r.set_body_poses(dev_poses[i])
            r.render(dev_cams[i], wl.fov, 1, **ekw, into=dev_out[i])
            rendered[i].record()
            if s + 1 < n:
                upload(s + 1)
            copier.wait_event(rendered[i])
            with torch.cuda.stream(copier):
                for k in shapes:
                    host_out[i][k].copy_(dev_out[i][k], non_blocking=True)
                copied[i].record()

    e2e_steps(2)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps(KE)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * views * KE / e2e_s
    out = host_out[0]
    h2d = pinned_poses[0].numel() * 4 + wl.cameras.nbytes
    d2h = sum(a.numel() * a.element_size() for a in out.values())

    # The other two forms of the metric, on the same GPU in the same run (one GPU only: they are single-GPU
    # figures): forward + backward against forward at 1024 worlds x 128x128, and the uneven batch.
    differentiable = uneven = None
    if rank == 0 and world == 1 and not args.no_forms:
        with ClockSampler(local_rank) as form_clocks:
            differentiable = differentiable_figures(dev, K, W)
            uneven = uneven_figures(dev, K, W)
        differentiable["clocks"] = uneven["clocks"] = form_clocks.summary()
    l2_gbs = l2_copy_gbs(torch, dev) if rank == 0 else None

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline(wl, steps_np, args.cpu_seconds)

    if rank != 0:
        return None
    peak, peak_kind = peaks()
    built = ng.build_meshes(d.meshes)
    blas_bytes = built["nodes"].nbytes + built["triangles"].nbytes
    b_img = algorithmic_bytes_per_image(wl, blas_bytes)
    alg = b_img * views
    rmed = statistics.median(render_ms)
    cam_ms = stage_ms[0]
    achieved = alg / (cam_ms / 1000.0) / 1e9
    counts = (cpu or {}).get("counts")
    rpi = counts["rays_per_image"] if counts else None
    tr = traffic_per_image()
    clk = clocks.summary()
    return {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": round(total_ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded body_worlds scene and random-walk poses)",
        "config": workload_config(args.worlds, {"parallelism": f"worlds sharded, {args.worlds} per GPU, no collective",
                                                "l2": "flushed between timed steps (256 MiB write)"}),
        "stages_ms": {"set_body_poses": round(statistics.median(build_ms), 4),
                      "render": round(rmed, 4),
                      **({"camera_rays": round(stage_ms[0], 4), "shading": round(stage_ms[1], 4),
                          "shadow_rays": round(stage_ms[2], 4)} if len(stage_ms) == 3 else {})},
        # Reference-equivalent work: the rays the reference's path traces per image and the bytes its walks fetch
        # (nodes, child-box pairs, instance inverses, triangles; almost all from L1/L2), as the oracle counts them
        # (it traces every shadow ray; this build leaves out those whose answer cannot change the pixel), at this
        # build's images/s, and that byte rate over the measured HBM peak (above 1 shows cache reuse).
        "reference_rays_per_s": None if rpi is None else round(value * rpi, 1),
        "reference_rays_per_image": None if rpi is None else round(rpi, 1),
        "traversal": None if not counts else {
            "bytes_per_image": round(counts["traversal_bytes_per_image"], 1),
            "achieved_gbs": round(counts["traversal_bytes_per_image"] * value / 1e9, 1),
            "l2_copy_gbs": round(l2_gbs, 1),
            "frac_of_l2_copy": round(counts["traversal_bytes_per_image"] * value / 1e9 / l2_gbs, 3),
            "what": "bytes the reference's walks fetch per image (32 per node, 64 per child-box pair, 48 per "
                    "instance inverse, 48 per triangle; the oracle's count) at this build's images/s, against "
                    "this GPU's copy bandwidth between two buffers resident in L2 (graph-captured copies), measured "
                    "in this run"},
        "e2e": {"value": round(e2e_value, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "steps": KE, "path": "pinned host poses and cameras -> device (copy on an upload stream while the step before "
                        "renders) -> BatchRenderer.set_body_poses + render(into= one of two device image sets) -> pinned host "
                        "images on a copy stream, overlapping the next step; host clock around all steps, the last copy out "
                        "included"},
        # The dominant kernel's launch carries the step's compulsory bytes (B_img per image, algorithmic_bytes_per
        # _image's terms) over its own CUDA-event duration; whole_step spreads them over the whole step instead.
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 5), "peak_kind": peak_kind,
                     "traffic": None if tr is None else int(tr * views),
                     "kernel": "camera_tiles_kernel", "kernel_ms": round(cam_ms, 4),
                     "algorithmic_bytes_per_image": round(b_img, 1), "algorithmic_bytes_per_launch": int(alg),
                     "whole_step": {"achieved": round(b_img * value / 1e9, 2),
                                    "frac": round(b_img * value / 1e9 / peak, 5)},
                     "issue": issue_figures()},
        "cpu_baseline": cpu,
        # Per step: the tree build (compose + per-world build, inter-world links) and the render: the camera-basis
        # kernel, the per-view candidate order and the camera, shade and shadow kernels (tile path), or the
        # camera-basis and one render kernel.
        "gpu_launches": (2 + (5 if len(stage_ms) == 3 else 2)) * K,
        "kernel_shape": None if tuned is None else {k: tuned[k] for k in ("kernel", "threads", "registers", "refill",
                                                                            "leaf_batch", "fetch", "paired", "ms")},
        # The renderers' own device arrays (scene, trees, per-pixel scratch; ngb_device_bytes), not the images.
        "device_mb": round(ng.device_bytes() / 1e6, 1),
        "differentiable": differentiable,
        "uneven": uneven,
        "clocks": clk,
    }


def run_large(args, rank, world, local_rank, dist):
    """One world of 100,000 instances: per frame, new instance matrices (device) -> global tree build ->
    1280x720 RGB + depth + ID -> LiDAR sweep of 131,072 rays. frames/s over the whole job, CUDA events.
    On N GPUs the one world is shared (strong scaling): rank 0's matrices are broadcast once, every rank
    builds the same tree, renders its band of 4-row tiles (ShardedFrame) and casts its share of the LiDAR
    rays (ShardedRays); the images and hits stay on their GPUs."""
    import torch

    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import workloads
    from neraulgraphics_b200.sharding import ShardedFrame, ShardedRays

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    K, W = args.steps, args.warmup
    wl = workloads.large_world(seed=0, frames=W + K)
    d = wl.desc
    r = ng.BatchRenderer(d.width, d.height, 1, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances, device=dev)
    mats = torch.from_numpy(wl.matrices).to(dev)
    cams = torch.from_numpy(wl.cameras).to(dev)
    lidar = wl.info["lidar"]
    lo, ld = torch.from_numpy(lidar["origins"]).to(dev), torch.from_numpy(lidar["directions"]).to(dev)
    frame_shard, ray_shard = ShardedFrame(d.height), ShardedRays(lo.shape[1])
    frame_shard.broadcast(mats)
    frame_shard.apply(r)
    lo_all, ld_all = lo, ld
    lo, ld = ray_shard.take(lo_all).contiguous(), ray_shard.take(ld_all).contiguous()
    kw = dict(rgb=True, depth=True, object_ids=True, zero_copy=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    r.set_instance_transforms(mats[0])
    tuned = None
    if not args.no_autotune:
        from neraulgraphics_b200.autotune import tune
        tuned = tune(r, cams, wl.fov, rgb=True, depth=True, object_ids=True, use_cache=False, budget_s=30.0)
    for s in range(W):
        r.set_instance_transforms(mats[s])
        r.render(cams, wl.fov, 1, **kw)
        r.cast_rays(lo, ld, lidar["max_distance"])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    with ClockSampler(local_rank) as clocks:
        for s in range(K):
            flush.zero_()
            e = ev[s]
            e[0].record()
            r.set_instance_transforms(mats[W + s])
            e[1].record()
            r.render(cams, wl.fov, 1, **kw)
            e[2].record()
            hits = r.cast_rays(lo, ld, lidar["max_distance"])
            e[3].record()
        torch.cuda.synchronize()
    stage = [[e[i].elapsed_time(e[i + 1]) for e in ev] for i in range(3)]
    total_ms = sum(sum(x) for x in stage)
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    hit_frac = float((hits["object_id"] > 0).float().mean())
    if rank != 0:
        return None
    rays = lo.shape[1]  # this rank's share (all of them on one GPU)
    return {
        "metric": "frames/s at 1 world x 100,000 instances, 1280x720 RGB+depth+ID + 64x2048 LiDAR, matrices redrawn "
                  "and tree rebuilt every frame",
        "value": round(K / (total_ms / 1000.0), 2), "unit": "frames/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": round(total_ms / K, 4), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded large_world scene)",
        "config": {"workload": "large_world: 1 world x 100,000 instances (box 12 / icosphere 320 / cylinder 512 / "
                               "icosphere 1280 / icosphere 20480 tris), 1280x720, 64x2048 LiDAR, max range 150",
                   "l2": "flushed between timed frames (256 MiB write)",
                   "split": f"rows {frame_shard.first}..{frame_shard.first + frame_shard.count - 1} and LiDAR rays "
                            f"{ray_shard.start}..{ray_shard.stop - 1} on rank 0 of {world}"},
        "stages_ms": {"set_instance_transforms": round(statistics.median(stage[0]), 4),
                      "render": round(statistics.median(stage[1]), 4),
                      "lidar": round(statistics.median(stage[2]), 4)},
        "step_ms": [round(stage[0][k] + stage[1][k] + stage[2][k], 3) for k in range(K)],
        "lidar_rays_per_s": round(rays / (statistics.median(stage[2]) / 1000.0), 1),
        "kernel_shape": None if tuned is None else {k: tuned[k] for k in ("kernel", "threads", "registers", "refill",
                                                                            "leaf_batch", "fetch", "paired", "ms")},
        "lidar_hit_fraction": round(hit_frac, 4),
        "clocks": clocks.summary(),
    }


def differentiable_figures(dev, K, W, seed=0, fd_world=3):
    """1024 worlds x 128x128, 12 instances: an L2 depth loss against a target rendered from perturbed poses.
    Forward only = poses -> matrices -> render depth + normals -> loss; forward + backward adds the hit
    records, the adjoint kernel and autograd back to positions, quaternions and cameras. Both timed per step
    with CUDA events (L2 flushed before each). The gradient is checked in the same run against central
    differences (h = 1e-3) of world fd_world's loss in float64, on its 12 instance positions and its camera
    position, with the target 0.5 nearer on pixels at least 2 px from a silhouette (every pixel's weight about
    1, so the float32 rounding of the rendered depths stays far below the differences)."""
    import torch

    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import workloads
    from neraulgraphics_b200.autodiff import pose_matrices, render_depth_normals

    wl = workloads.differentiable_worlds(worlds=1024, seed=seed)
    d, info = wl.desc, wl.info
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device=dev)
    T = lambda a: torch.from_numpy(a).to(dev)
    pos, quat, scale, cams = T(info["positions"]), T(info["quaternions"]), T(info["scales"]), T(wl.cameras)
    with torch.no_grad():
        target = render_depth_normals(r, pose_matrices(T(info["target_positions"]), T(info["target_quaternions"]),
                                                       scale), cams, wl.fov)[0].clone()
    ok = torch.isfinite(target)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def forward():
        with torch.no_grad():
            r.set_instance_transforms(pose_matrices(pos, quat, scale).contiguous())
            out = r.render(cams, wl.fov, 1, rgb=False, depth=True, normals=True, zero_copy=True)
            dep = out["depth"]
            return (torch.where(ok & torch.isfinite(dep), dep - target, 0.0) ** 2).sum()

    p, q, c = pos.clone().requires_grad_(), quat.clone().requires_grad_(), cams.clone().requires_grad_()

    def forward_backward():
        p.grad = q.grad = c.grad = None
        dep = render_depth_normals(r, pose_matrices(p, q, scale), c, wl.fov)[0]
        loss = (torch.where(ok & torch.isfinite(dep), dep - target, 0.0) ** 2).sum()
        loss.backward()
        return loss

    def timed(fn):
        for _ in range(W):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(K):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    fwd_ms = timed(forward)
    fb_ms = timed(forward_backward)
    r.set_instance_transforms(pose_matrices(pos, quat, scale).detach().contiguous())
    forward_backward()
    adj_ms = r.last_kernel_ms

    # Central differences of world fd_world's conditioned loss.
    w = fd_world
    with torch.no_grad():
        base = render_depth_normals(r, pose_matrices(pos, quat, scale), cams, wl.fov)[0][w].clone()
    ids = r.render(cams, wl.fov, 1, rgb=False, object_ids=True, zero_copy=True)["object_ids"][w]
    edge = torch.zeros_like(ids, dtype=torch.bool)
    edge[1:, :] |= ids[1:, :] != ids[:-1, :]
    edge[:-1, :] |= ids[1:, :] != ids[:-1, :]
    edge[:, 1:] |= ids[:, 1:] != ids[:, :-1]
    edge[:, :-1] |= ids[:, 1:] != ids[:, :-1]
    near_edge = torch.nn.functional.max_pool2d(edge[None, None].float(), 5, 1, 2)[0, 0] > 0
    mask = ~near_edge & torch.isfinite(base)
    nearer = torch.where(mask, base - 0.5, 0.0)

    def world_loss(pp, qq, cc, grad=False):
        dep = render_depth_normals(r, pose_matrices(pp, qq, scale), cc, wl.fov)[0][w]
        value = (torch.where(mask, dep - nearer, 0.0).double() ** 2).sum()
        return value if grad else float(value)

    p.grad = q.grad = c.grad = None
    world_loss(p, q, c, grad=True).backward()
    h = 1e-3
    got, fd = [], []
    with torch.no_grad():
        for i in range(d.per_world):
            for k in range(3):
                plus, minus = pos.clone(), pos.clone()
                plus[w, i, k] += h
                minus[w, i, k] -= h
                fd.append((world_loss(plus, quat, cams) - world_loss(minus, quat, cams)) / (2 * h))
                got.append(float(p.grad[w, i, k]))
        for k in range(3):
            plus, minus = cams.clone(), cams.clone()
            plus[w, k, 3] += h
            minus[w, k, 3] -= h
            fd.append((world_loss(pos, quat, plus) - world_loss(pos, quat, minus)) / (2 * h))
            got.append(float(c.grad[w, k, 3]))
    got, fd = np.array(got), np.array(fd)
    err = float(np.linalg.norm(got - fd) / max(np.linalg.norm(fd), 1e-30))
    views = d.view_count
    return {"forward_ms": round(fwd_ms, 4), "forward_backward_ms": round(fb_ms, 4),
            "ratio": round(fb_ms / fwd_ms, 4), "adjoint_kernel_ms": round(adj_ms, 4),
            "forward_images_per_s": round(views / (fwd_ms / 1000.0), 1),
            "forward_backward_images_per_s": round(views / (fb_ms / 1000.0), 1),
            "gradient_rel_err": round(err, 6),
            "gradient_check": f"central differences (h = 1e-3) of world {w}'s float64 loss on its {d.per_world} "
                              f"instance positions and its camera position ({len(got)} parameters); the tests add "
                              "a float64 CPU restatement of the gradient on sampled worlds",
            "workload": "differentiable_worlds: 1024 worlds x 12 instances (icosphere 1280 / box 12 tris), 128x128, "
                        "depth+normals, L2 depth loss against a target rendered from poses perturbed by N(0, 0.01) "
                        "position and 0.02 rad rotation"}


def run_differentiable(args, rank, world, local_rank, dist):
    """The differentiable form alone (differentiable_figures): forward + backward over forward-only time."""
    import torch

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    K, W = args.steps, args.warmup
    with ClockSampler(local_rank) as clocks:
        f = differentiable_figures(dev, K, W, seed=rank)
    if rank != 0:
        return None
    return {
        "metric": "forward+backward time / forward-only time at 1024 worlds x 128x128 depth+normals (L2 depth loss)",
        "value": f["ratio"], "unit": "ratio", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": f["forward_backward_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded differentiable_worlds scene and perturbed target poses)",
        "config": {"workload": f["workload"], "l2": "flushed before every timed step (256 MiB write)"},
        **{k: v for k, v in f.items() if k not in ("ratio", "workload")},
        "clocks": clocks.summary(),
    }


def uneven_figures(dev, K, W, seed=0, buckets=False):
    """2048 worlds of 1..200 instances at 32x32, 64x64 or 128x128, RGB + depth + ID. Per step the instance
    matrices of the random walk go to the device (one copy into the graph's input), then one CUDA graph
    replays the whole step: the tree build of every world and the render of every view (camera, shade and
    shadow kernels). With buckets, also the same steps through plain renderers, one per (resolution, instance
    count) bucket, launched one after another."""
    import torch

    import neraulgraphics_b200 as ng
    from neraulgraphics_b200 import workloads
    from neraulgraphics_b200.autotune import tune

    wl = workloads.uneven_worlds(seed=seed)
    mats = torch.from_numpy(workloads.walk_uneven(wl, W + K, seed=1 + seed)).to(dev)
    cams = torch.from_numpy(wl["cameras"]).to(dev)
    r = ng.UnevenBatchRenderer(wl["worlds"], lights=wl["lights"], floor=wl["floor"], meshes=wl["meshes"], device=dev)
    kw = dict(rgb=True, depth=True, object_ids=True, zero_copy=True)
    static = mats[0].clone()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    r.set_instance_transforms(static)
    tuned = tune(r, cams, wl["fov"], rgb=True, depth=True, object_ids=True, use_cache=False)
    # One graph for the whole step, captured after warm-up renders on the capture stream.
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            r.set_instance_transforms(static)
            r.render(cams, wl["fov"], 1, **kw)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        r.set_instance_transforms(static)
        out = r.render(cams, wl["fov"], 1, **kw)
    # The graph's images equal an eager render's, after a pose change.
    static.copy_(mats[1])
    graph.replay()
    torch.cuda.synchronize()
    from_graph = {k: v.clone() for k, v in out.items()}
    r.set_instance_transforms(mats[1].clone())
    eager = r.render(cams, wl["fov"], 1, **kw)
    same = all(bool(torch.equal(from_graph[k], eager[k])) for k in from_graph)

    def timed(step):
        for s in range(W):
            step(s)
        torch.cuda.synchronize()
        ms = []
        for s in range(K):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            step(W + s)
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    def graph_step(s):
        static.copy_(mats[s])
        graph.replay()

    graph_ms = timed(graph_step)
    views = len(wl["worlds"])
    first = r.instance_first
    res = {"images_per_s": round(views / (graph_ms / 1000.0), 1), "ms_per_step": round(graph_ms, 4),
           "kernel_shape": {k: tuned[k] for k in tuned if k != "timings"},
           "shape_timings_ms": {f"{t['threads']}/{t['registers']} fetch {t['fetch']} "
                                f"{'paired' if t['paired'] else 'one kind'}": round(t["ms"], 4)
                                for t in tuned["timings"]},
           "graph_matches_eager": same, "gpu_launches_per_step": 7,
           "workload": f"uneven_worlds: {views} worlds, {int(first[-1])} instances, {r.pixel_count} pixels; six "
                       "meshes of 12 to 20480 triangles; one light, spp 1, RGB+depth+ID"}
    if not buckets:
        return res
    groups = {}
    for w, (size, _, insts) in enumerate(wl["worlds"]):
        groups.setdefault((size, len(insts)), []).append(w)
    plain = []
    for (size, count), ws in sorted(groups.items()):
        insts = wl["worlds"][ws[0]][2]
        rb = ng.BatchRenderer(size, size, len(ws), 1, [], wl["lights"], wl["floor"], wl["meshes"], insts, device=dev)
        idx = torch.from_numpy(np.concatenate([np.arange(first[w], first[w + 1]) for w in ws])).to(dev)
        plain.append((rb, mats[:, idx].contiguous(), cams[torch.tensor(ws, device=dev)].contiguous()))

    def plain_step(s):
        for rb, mb, cb in plain:
            rb.set_instance_transforms(mb[s])
            rb.render(cb, wl["fov"], 1, **kw)

    plain_ms = timed(plain_step)
    res["bucketed_plain"] = {"value": round(views / (plain_ms / 1000.0), 1), "unit": "images/s",
                             "ms_per_step": round(plain_ms, 4), "buckets": len(plain),
                             "what": "one plain BatchRenderer per (resolution, instance count) bucket, set_instance_"
                                     "transforms + render each, launched one after another"}
    return res


def run_uneven(args, rank, world, local_rank, dist):
    """The uneven form alone (uneven_figures), against bucketed plain renderers."""
    import torch

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    K, W = args.steps, args.warmup
    with ClockSampler(local_rank) as clocks:
        f = uneven_figures(dev, K, W, seed=rank, buckets=True)
    if rank != 0:
        return None
    return {
        "metric": "images/s at 2048 uneven worlds (1..200 instances, 32/64/128 px) RGB+depth+ID, one CUDA graph per "
                  "step (tree build + render)",
        "value": round(world * f["images_per_s"], 1), "unit": "images/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": f["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uneven_worlds scene and random-walk poses)",
        "config": {"workload": f["workload"], "l2": "flushed before every timed step (256 MiB write)"},
        **{k: v for k, v in f.items() if k not in ("images_per_s", "ms_per_step", "workload")},
        "clocks": clocks.summary(),
    }


def reference_cuda_large(wl, torch, mats, cams, lo, ld, steps, warmup):
    """The reference's CUDA backend on the same large-world frames, inputs on the device: ms per stage."""
    import oracle as O
    if not O.reference_available(cuda=True):
        return None
    ref = O.Reference(wl.desc, cuda=True)
    lidar = wl.info["lidar"]
    stream = torch.cuda.default_stream()
    for s in range(warmup):
        ref.set_instance_transforms(mats[s].data_ptr(), device=True)
        ref.render_device(cams.data_ptr(), wl.fov, 1, 1 | 2 | 8)
        ref.cast_rays_device(lo.data_ptr(), ld.data_ptr(), lo.shape[1], lidar["max_distance"])
    torch.cuda.synchronize()
    stage = [[], [], []]
    for s in range(steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(stream)
        ref.set_instance_transforms(mats[warmup + s].data_ptr(), device=True)
        e[1].record(stream)
        ref.render_device(cams.data_ptr(), wl.fov, 1, 1 | 2 | 8)
        e[2].record(stream)
        ref.cast_rays_device(lo.data_ptr(), ld.data_ptr(), lo.shape[1], lidar["max_distance"])
        e[3].record(stream)
        e[3].synchronize()
        for i in range(3):
            stage[i].append(e[i].elapsed_time(e[i + 1]))
    ms = [statistics.median(x) for x in stage]
    return {"value": round(1000.0 / sum(ms), 2), "unit": "frames/s",
            "stages_ms": {"set_instance_transforms": round(ms[0], 4), "render": round(ms[1], 4), "lidar": round(ms[2], 4)},
            "what": "neraulgraphics 0.5.0 CudaBackend, same frames on the device, median step"}


def run_mesh_update(args, rank, world, local_rank, dist):
    """Meshes whose vertices move: the five meshes of the large world (12, 320, 512, 1280 and 20,480
    triangles) get new vertex positions every step (a twist and a stretch that change from step to step), each
    mesh's tree is rebuilt on the GPU (update_mesh: the host's binned SAH build, node for node) and the instance
    trees of 64 worlds x 5 instances are rebuilt around the meshes' new boxes. `value`: vertices already on the
    GPU; `e2e`: vertices from pinned host memory. Timed on the host clock around synchronised steps (the rebuild
    reads each tree level's size back), with CUDA events beside it. The reference changes a mesh only by
    building a new renderer, whose host build_meshes (src/mesh_build.cpp:91-157) is timed here on the same
    vertices (cpu_baseline)."""
    import torch

    import neraulgraphics_b200 as ng
    import oracle as O
    from neraulgraphics_b200 import scene as S
    from neraulgraphics_b200 import workloads

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    K, W = args.steps, args.warmup
    base = workloads.large_world(instances=5).desc.meshes
    worlds = 64
    insts = [S.Instance(i, S.make_transform((2.0 * i - 4.0, 0.0, -6.0), (0, 0, 0, 1), 1.0)) for i in range(5)]
    r = ng.BatchRenderer(64, 64, worlds, 1, [], [workloads.LIGHT], None, base, insts, device=dev)

    def shape(mesh, step):
        v = mesh.vertices.astype(np.float64)
        a = (0.2 + 0.05 * step) * v[:, 1]
        x = v[:, 0] * np.cos(a) - v[:, 2] * np.sin(a)
        z = v[:, 0] * np.sin(a) + v[:, 2] * np.cos(a)
        return np.stack([(1.0 + 0.02 * step) * x, v[:, 1], z], 1).astype(np.float32)

    steps = [[shape(m, s) for m in base] for s in range(W + K)]
    on_dev = [[torch.from_numpy(v).to(dev) for v in st] for st in steps]
    pinned = [[torch.from_numpy(v).pin_memory() for v in st] for st in steps]

    def run(arrays):
        for s in range(W):
            for m, v in enumerate(arrays[s]):
                r.update_mesh(m, v)
        torch.cuda.synchronize()
        host_ms, dev_ms = [], []
        for s in range(W, W + K):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            for m, v in enumerate(arrays[s]):
                r.update_mesh(m, v)
            e1.record()
            torch.cuda.synchronize()
            host_ms.append(1000.0 * (time.perf_counter() - t0))
            dev_ms.append(e0.elapsed_time(e1))
        return statistics.median(host_ms), statistics.median(dev_ms)

    with ClockSampler(local_rank) as clocks:
        host_ms, dev_ms = run(on_dev)
        e2e_ms, _ = run([[t.numpy() for t in st] for st in pinned])
    node_ok = all(np.array_equal(r.inspect_mesh(i)["nodes"], ng.build_meshes([S.Mesh(v, m.triangles)])["nodes"])
                  for i, (v, m) in enumerate(zip(steps[-1], base)))
    if rank != 0:
        return None
    cpu = None
    if O.reference_available():
        ref_ms = []
        for s in range(min(K, 10)):
            t0 = time.perf_counter()
            O.ref_build_meshes([S.Mesh(v, m.triangles) for v, m in zip(steps[W + s], base)])
            ref_ms.append(1000.0 * (time.perf_counter() - t0))
        cpu = {"value": round(statistics.median(ref_ms), 4), "unit": "ms per step", "cores": 1, "kind": "reference",
               "sample": "the reference's build_meshes (host, one thread) of the same five moved meshes, "
                         f"median of {len(ref_ms)} steps"}
    tris = sum(len(m.triangles) for m in base)
    return {
        "metric": f"ms per step: five mesh trees ({tris} triangles, 12 to 20,480 per mesh) rebuilt from new vertex "
                  "positions, then the instance trees of 64 worlds",
        "value": round(host_ms, 4), "unit": "ms per step", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": round(host_ms, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (the large world's five meshes, twisted and stretched per step)",
        "config": {"workload": "mesh_update: box 12, icosphere s2 320, cylinder 512, icosphere s3 1280, icosphere s5 "
                               "20480 triangles; 64 worlds x 5 instances", "l2": "inputs of 0.5 MB: L2 not flushed"},
        "device_ms_per_step": round(dev_ms, 4),
        "trees_equal_host_build": bool(node_ok),
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms per step",
                "h2d_bytes_per_step": int(sum(v.nbytes for v in steps[0])), "d2h_bytes_per_step": 0},
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }


def reference_cuda_arm(run, what):
    """run(torch) on cuda:0 when a GPU is present: the reference's own CUDA backend (built from its sources into
    oracle/_ref) timed on the same workload, reported beside the reference arm's CPU figure."""
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
        torch.cuda.set_device(0)
        out = run(torch)
        return out if out is not None else {"unavailable": f"oracle/_ref was built without CUDA ({what})"}
    except Exception as e:  # reported, not fatal: the CPU figure is the arm's value
        return {"unavailable": f"{type(e).__name__}: {e}"}


def run_reference(args, rank):
    """The reference's own CPU implementation, rank 0 only, with every host core; and, beside it, the reference's
    CUDA backend on the GPU on the same workload (reference_cuda)."""
    from neraulgraphics_b200 import workloads
    import oracle as O
    if rank != 0:
        return None
    if not O.reference_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libngref.so is not built (make -C oracle ref)"}
    if args.config == "large_world":
        return run_reference_large(args)
    if args.config != "body_worlds":
        return {"impl": "reference", "unavailable": f"--config {args.config} has no reference arm: the reference "
                "has no gradients, no uneven worlds and no device mesh build (its host build is this config's "
                "cpu_baseline)"}
    from neraulgraphics_b200.scene import SceneDesc
    wl = workloads.body_worlds(worlds=args.worlds, seed=0)
    sample = 64
    steps_np = workloads.random_walk(wl.poses[:sample], args.warmup + args.steps, seed=1)
    d = wl.desc
    desc = SceneDesc(d.width, d.height, sample, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances)
    cores = os.cpu_count() or 1
    ref = O.Reference(desc, threads=cores)
    ref.bind_bodies(**wl.binding)
    cams = wl.cameras[:sample]
    for s in range(args.warmup):
        ref.set_body_poses(steps_np[s])
        ref.render(cams, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    t0 = time.perf_counter()
    for s in range(args.steps):
        ref.set_body_poses(steps_np[args.warmup + s])
        ref.render(cams, wl.fov, 1, rgb=True, depth=True, object_ids=True)
    el = time.perf_counter() - t0
    value = sample * args.steps / el
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * el / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded body_worlds scene and random-walk poses)",
        "config": workload_config(args.worlds, {"sample": f"{sample} of the {args.worlds} worlds per step"}),
        "cpu_baseline": {"value": round(value, 2), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{sample} worlds per step, {args.steps} steps, neraulgraphics 0.5.0 CPU backend"},
        "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": None if args.no_reference_cuda else reference_cuda_arm(
            lambda torch: reference_cuda_body(args, torch), "body_worlds"),
    }


def reference_cuda_body(args, torch):
    """The reference's CUDA backend on the whole body_worlds workload: the same seeded poses and cameras on the
    device as the other arm's timed steps."""
    from neraulgraphics_b200 import workloads
    wl = workloads.body_worlds(worlds=args.worlds, seed=0)
    K, W = min(args.steps, 10), min(args.warmup, 3)
    poses = torch.from_numpy(workloads.random_walk(wl.poses, W + K, seed=1)).cuda()
    cams = torch.from_numpy(wl.cameras).cuda()
    return reference_cuda(wl, torch, poses, cams, K, W)


def run_reference_large(args):
    """The reference's CPU backend on the large world (one world of 100,000 instances: matrices in, its host
    tree build, 1280x720 RGB+depth+ID, the 64x2048 LiDAR sweep), every host core, on a bounded sample of each
    frame: a full frame takes it about ten minutes (0.7 ms per pixel, 0.8 ms per LiDAR ray on 8 cores), so it
    renders the frame at 64x36 (the same camera and aspect, 1/400 of the pixels) and casts every 128th LiDAR
    ray, and the frame's time is extrapolated from those per-pixel and per-ray costs. Its CUDA backend runs
    the whole frames on the GPU."""
    from neraulgraphics_b200 import workloads
    from neraulgraphics_b200.scene import SceneDesc
    import oracle as O
    K, W = min(args.steps, 2), min(args.warmup, 1)
    wl = workloads.large_world(seed=0, frames=W + K)
    d = wl.desc
    lidar = wl.info["lidar"]
    cores = os.cpu_count() or 1
    sw, sh, every = 64, 36, 128
    small = SceneDesc(sw, sh, 1, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances)
    ref = O.Reference(small, threads=cores)
    lo_s = np.ascontiguousarray(lidar["origins"][:, ::every])
    ld_s = np.ascontiguousarray(lidar["directions"][:, ::every])
    pixel_scale = (d.width * d.height) / (sw * sh)
    ray_scale = lidar["origins"].shape[1] / lo_s.shape[1]
    frame_s = []
    for s in range(W + K):
        t0 = time.perf_counter()
        ref.set_instance_transforms(wl.matrices[s])
        t1 = time.perf_counter()
        ref.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, object_ids=True)
        t2 = time.perf_counter()
        ref.cast_rays(lo_s, ld_s, lidar["max_distance"])
        t3 = time.perf_counter()
        if s >= W:
            frame_s.append((t1 - t0) + (t2 - t1) * pixel_scale + (t3 - t2) * ray_scale)
    value = 1.0 / statistics.median(frame_s)

    def cuda(torch):
        mats = torch.from_numpy(wl.matrices).cuda()
        cams = torch.from_numpy(wl.cameras).cuda()
        lo, ld = torch.from_numpy(lidar["origins"]).cuda(), torch.from_numpy(lidar["directions"]).cuda()
        return reference_cuda_large(wl, torch, mats, cams, lo, ld, K, W)

    return {
        "impl": "reference", "metric": "frames/s at 1 world x 100,000 instances, 1280x720 RGB+depth+ID + 64x2048 "
        "LiDAR, matrices redrawn and tree rebuilt every frame", "value": round(value, 6), "unit": "frames/s",
        "n_gpus": args.gpus, "steps": K, "warmup": W, "ms_per_step": round(1000 / value, 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded large_world scene)",
        "config": {"workload": "large_world: 1 world x 100,000 instances, 1280x720, 64x2048 LiDAR, max range 150"},
        "cpu_baseline": {"value": round(value, 6), "unit": "frames/s", "cores": cores, "kind": "reference",
                         "sample": f"{K} frames after {W} warm-up, neraulgraphics 0.5.0 CPU backend: "
                                   f"set_instance_transforms in full, render_host at {sw}x{sh} (x{pixel_scale:.0f}) "
                                   f"and every {every}th LiDAR ray (x{ray_scale:.0f}), extrapolated to whole frames"},
        "e2e": {"value": round(value, 6), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": None if args.no_reference_cuda else reference_cuda_arm(cuda, "large_world"),
    }


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if args.impl == "reference":
        line = run_reference(args, rank)
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device(f"cuda:{local_rank}"))
        run = {"body_worlds": run_ours, "large_world": run_large, "differentiable": run_differentiable,
               "uneven": run_uneven, "mesh_update": run_mesh_update}[args.config]
        line = run(args, rank, world, local_rank, dist)
        if dist:
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
