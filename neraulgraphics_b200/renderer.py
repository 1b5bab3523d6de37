"""BatchRenderer: the reference's Python class (python/bindings.cpp:667-799), over the C ABI.

Arrays may be NumPy arrays (host: checked, then copied) or CUDA tensors from PyTorch (device: used where
they are, on PyTorch's current stream, unchecked, as in the reference). With zero_copy=True the images
come back as CUDA tensors that alias the renderer's own buffers, overwritten by the next render; work is
queued on PyTorch's current stream, so PyTorch code on that stream sees it in order. Otherwise they come
back as NumPy copies.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi
from ._lib import CudaError, check, lib
from .scene import Environment, Plane, SceneDesc, lights_abi

_TIMEOUT_S = 120.0


def _torch():
    import torch  # plumbing only: device memory and streams
    return torch


def _is_cuda_tensor(a) -> bool:
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


def _cuda_view(a):
    """A CUDA tensor over a's memory when a is a CUDA array of another library (a Warp, CuPy or Numba array:
    anything with __cuda_array_interface__), so that a simulator's arrays are read in place; else a itself."""
    if not _is_cuda_tensor(a) and hasattr(a, "__cuda_array_interface__"):
        return _torch().as_tensor(a)
    return a


def _count(a) -> int:
    return int(np.prod(a.shape)) if len(a.shape) else 1


def _require_count(a, expected, what, shape):
    if _count(a) != expected:
        raise ValueError(f"{what} has {_count(a)} values, but {expected} are needed: {shape}")


def _parse_device(device) -> int:
    if device in ("auto", "cuda", None):
        return 0
    if isinstance(device, int):
        return device
    if isinstance(device, str) and device.startswith("cuda:"):
        return int(device.split(":", 1)[1])
    if device == "cpu":
        raise ValueError("device 'cpu' is not available: this renderer runs on CUDA GPUs only")
    raise ValueError(f"device must be 'auto', 'cuda' or 'cuda:N', got '{device}'")


class BatchRenderer:
    """Many worlds rendered at once: thousands of copies of one environment, each seen by its own camera(s).

    All worlds share the meshes, lights, spheres and floor. Each holds the same list of instances, placed
    differently, and a camera sees only its own world's. Views are numbered world-major: view v looks at
    world v // cameras_per_world.
    """

    def __init__(self, width, height, world_count, cameras_per_world=1, spheres=(), lights=(), floor=None,
                 meshes=(), instances=(), textures=(), device="auto"):
        if textures:
            raise ValueError("textures are not supported by this renderer")
        self._device = _parse_device(device)
        self._desc = SceneDesc(width, height, world_count, cameras_per_world, spheres, lights,
                               floor if floor is not None else Plane(), meshes, instances, self._device)
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.ngb_create(C.byref(self._desc.c), C.byref(h)), None)
        self._h = h
        # Stream-ordered on PyTorch's current stream.
        check(self._lib.ngb_set_sync(self._h, 0, _TIMEOUT_S), self._h)
        self._out = {}
        self._rays = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.ngb_destroy(h)
            self._h = None

    # ------------------------------------------------------------------------------------------- plumbing --

    def _stream(self):
        torch = _torch()
        s = torch.cuda.current_stream(self._device).cuda_stream
        # PyTorch's default stream is CUDA's legacy default stream, handle 0; the C ABI takes NULL as the
        # renderer's own stream, so the legacy stream is named by its CUDA handle, cudaStreamLegacy (0x1).
        check(self._lib.ngb_set_stream(self._h, C.c_void_p(s if s else 1)), self._h)

    def _input(self, a, what):
        """(pointer, memory, keep-alive) for a float32 input: a CUDA array in place, else a host copy."""
        a = _cuda_view(a)
        if _is_cuda_tensor(a):
            torch = _torch()
            if a.device.index != self._device:
                raise ValueError(f"{what} is on cuda:{a.device.index}, but the renderer is on cuda:{self._device}")
            t = a if (a.dtype == torch.float32 and a.is_contiguous()) else a.to(torch.float32).contiguous()
            return C.c_void_p(t.data_ptr()), _abi.MEMORY_DEVICE, t
        if type(a).__module__.startswith("torch"):
            a = a.numpy()
        arr = np.ascontiguousarray(a, dtype=np.float32)
        return arr.ctypes.data_as(C.c_void_p), _abi.MEMORY_HOST, arr

    # ----------------------------------------------------------------------------------------- placement --

    def set_instance_transforms(self, matrices):
        """Place every instance of every world: (world_count, instances_per_world, 3, 4) float32."""
        expected = self.world_count * self.instances_per_world * 12
        _require_count(matrices, expected, "matrices",
                       "(world_count, instances_per_world, 3, 4), the top three rows of each 4x4")
        p, mem, keep = self._input(matrices, "matrices")
        self._stream()
        check(self._lib.ngb_set_instance_transforms(self._h, p, mem), self._h)
        self._keep = keep

    def bind_bodies(self, body_of_instance, local_pose, scale, bodies_per_world):
        """How simulator bodies carry the instances (per instance: body or -1, x y z qx qy qz qw, scale xyz)."""
        b = np.ascontiguousarray(body_of_instance, np.int32)
        lp = np.ascontiguousarray(local_pose, np.float32)
        sc = np.ascontiguousarray(scale, np.float32)
        n = self.instances_per_world
        if b.size != n or lp.size != 7 * n or sc.size != 3 * n:
            raise ValueError(f"a body binding needs one body index, 7 pose floats and 3 scale floats for each of the "
                             f"{n} instances of a world")
        self._stream()
        check(self._lib.ngb_bind_bodies(self._h, int(bodies_per_world), b.ctypes.data_as(C.POINTER(C.c_int32)),
                                        lp.ctypes.data_as(C.POINTER(C.c_float)),
                                        sc.ctypes.data_as(C.POINTER(C.c_float))), self._h)
        self._bodies_per_world = int(bodies_per_world)
        self._geoms_per_world = None

    def set_body_poses(self, body_poses):
        """Place every instance from body poses: (world_count, bodies_per_world, 7) floats, x y z qx qy qz qw."""
        p, mem, keep = self._input(body_poses, "body poses")
        bpw = getattr(self, "_bodies_per_world", None)
        body_poses = _cuda_view(body_poses)
        if bpw is not None:
            _require_count(body_poses, self.world_count * bpw * 7, "body poses", "(world_count, bodies_per_world, 7)")
        self._stream()
        check(self._lib.ngb_set_body_poses(self._h, p, mem), self._h)
        self._keep = keep

    def bind_geoms(self, geom_of_instance, scale, geoms_per_world):
        """How a MuJoCo model's geoms carry the instances: per instance its geom index and scale (x, y, z), as
        MJWarpBatchRenderer keeps them (python/neraulgraphics/mujoco.py:199-243). Replaces a body binding."""
        g = np.ascontiguousarray(geom_of_instance, np.int32)
        sc = np.ascontiguousarray(scale, np.float32)
        n = self.instances_per_world
        if g.size != n or sc.size != 3 * n:
            raise ValueError(f"a geom binding needs one geom index and 3 scale floats for each of the {n} instances "
                             f"of a world")
        self._stream()
        check(self._lib.ngb_bind_geoms(self._h, int(geoms_per_world), g.ctypes.data_as(C.POINTER(C.c_int32)),
                                       sc.ctypes.data_as(C.POINTER(C.c_float))), self._h)
        self._geoms_per_world = int(geoms_per_world)
        self._bodies_per_world = None

    def set_geom_poses(self, geom_xpos, geom_xmat):
        """Place every instance from its geom's pose, as a MuJoCo Warp data holds them: geom_xpos
        (world_count, geoms_per_world, 3) and geom_xmat (world_count, geoms_per_world, 3, 3) floats, read in
        place when they are CUDA arrays. Composes [R * diag(scale) | p] and rebuilds the trees in one launch
        (MJWarpBatchRenderer.update, python/neraulgraphics/mujoco.py:304-314)."""
        gpw = getattr(self, "_geoms_per_world", None)
        if gpw is None:
            raise ValueError("set_geom_poses needs bind_geoms to be called first")
        _require_count(geom_xpos, self.world_count * gpw * 3, "geom_xpos", "(world_count, geoms_per_world, 3)")
        _require_count(geom_xmat, self.world_count * gpw * 9, "geom_xmat", "(world_count, geoms_per_world, 3, 3)")
        p, mem_p, keep_p = self._input(geom_xpos, "geom_xpos")
        r, mem_r, keep_r = self._input(geom_xmat, "geom_xmat")
        if mem_p != mem_r:
            raise ValueError("geom_xpos and geom_xmat must both be CUDA arrays or both host arrays")
        self._stream()
        check(self._lib.ngb_set_geom_poses(self._h, p, r, mem_p), self._h)
        self._keep = (keep_p, keep_r)

    def update_mesh(self, mesh, vertices, normals=None):
        """New vertex positions for mesh `mesh` (the vertex count and triangles it was made with): (V, 3) floats,
        host or CUDA, and optionally new vertex normals. Its tree is rebuilt on the GPU as the renderer's
        construction builds it on the host (src/bvh.cpp:46-174), node for node, and every world's instance tree
        is rebuilt from the current transforms."""
        p, mem, keep = self._input(vertices, "vertices")
        pn = None
        if normals is not None:
            pn, mem_n, keep_n = self._input(normals, "normals")
            if mem_n != mem:
                raise ValueError("vertices and normals must both be CUDA arrays or both host arrays")
            if _count(normals) != _count(vertices):
                raise ValueError(f"normals has {_count(normals)} values, but vertices has {_count(vertices)}")
        m = self._desc.meshes[mesh] if 0 <= mesh < len(self._desc.meshes) else None
        if m is not None and _count(vertices) != m.vertices.size:
            raise ValueError(f"mesh {mesh} has {len(m.vertices)} vertices, but {_count(vertices)} values were given "
                             f"({len(m.vertices)} x 3 are needed)")
        self._stream()
        check(self._lib.ngb_update_mesh(self._h, int(mesh), p, pn, mem), self._h)
        self._keep = keep

    def inspect_mesh(self, mesh) -> dict:
        """Mesh `mesh`'s tree as the renderer holds it now, in build_meshes's format for that mesh alone."""
        nn, nt = C.c_int32(), C.c_int32()
        check(self._lib.ngb_inspect_mesh(self._h, int(mesh), C.byref(nn), C.byref(nt), None, None, None, None), self._h)
        nodes = np.zeros((nn.value, 8), np.int32)
        tris = np.zeros((nt.value, 12), np.float32)
        bounds = np.zeros((1, 6), np.float32)
        tidx = np.zeros(nt.value, np.int32)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(self._lib.ngb_inspect_mesh(self._h, int(mesh), C.byref(nn), C.byref(nt), vp(nodes), vp(tris), vp(bounds),
                                         vp(tidx)), self._h)
        return {"nodes": nodes, "triangles": tris, "roots": np.zeros(1, np.int32), "bounds": bounds,
                "triangle_index": tidx}

    # ------------------------------------------------------------------------------------------ rendering --

    def _buffer(self, key, shape, dtype):
        torch = _torch()
        t = self._out.get(key)
        if t is None or tuple(t.shape) != shape:
            t = torch.empty(shape, dtype=dtype, device=f"cuda:{self._device}")
            self._out[key] = t
        return t

    def render(self, cameras, fov=1.0, samples_per_pixel=1, *, rgb=True, depth=False, normals=False,
               object_ids=False, frame=0, zero_copy=False, out=None, into=None):
        """Render every view; returns a dict of 'rgb' (V,H,W,3) uint8, 'depth' (V,H,W) float32, 'normals'
        (V,H,W,3) float32, 'object_ids' (V,H,W) int32, for the images asked for (H: the rows drawn, set_rows).

        out: optional dict of preallocated host (NumPy) arrays, pinned or not, to copy the images into
        (BatchRenderer::render_host, src/batch.cpp:164-178); cameras must then be on the host.
        into: optional dict of the caller's CUDA tensors (contiguous, those shapes and dtypes, on the renderer's
        device) to render into instead of the renderer's own buffers, queued on PyTorch's current stream (as
        zero_copy): the caller may then copy them out while the next render runs."""
        torch = _torch()
        views, h, w = self.view_count, self.rows[1], self.width
        if out is not None:
            return self._render_host(cameras, fov, samples_per_pixel, rgb, depth, normals, object_ids, frame, out)
        _require_count(cameras, views * 12, "cameras", f"{views} cameras of 3 x 4 numbers (camera-to-world)")
        if into is not None:
            zero_copy = True
        if not zero_copy and _is_cuda_tensor(cameras):
            raise ValueError("cameras on the GPU need zero_copy=True: the results then stay on the GPU too")
        outputs = ((_abi.OUTPUT_RGB if rgb else 0) | (_abi.OUTPUT_DEPTH if depth else 0) |
                   (_abi.OUTPUT_NORMAL if normals else 0) | (_abi.OUTPUT_OBJECT_ID if object_ids else 0))
        want = {"rgb": ((views, h, w, 3), torch.uint8, rgb), "depth": ((views, h, w), torch.float32, depth),
                "normals": ((views, h, w, 3), torch.float32, normals),
                "object_ids": ((views, h, w), torch.int32, object_ids)}
        bufs = {}
        for k, (shape, dtype, on) in want.items():
            if not on:
                continue
            if into is None:
                bufs[k] = self._buffer(k, shape, dtype)
                continue
            t = into.get(k)
            if (t is None or not _is_cuda_tensor(t) or tuple(t.shape) != shape or t.dtype != dtype or
                    not t.is_contiguous() or t.device.index != self._device):
                raise ValueError(f"into['{k}'] must be a contiguous {dtype} CUDA tensor of shape {shape} on "
                                 f"cuda:{self._device}")
            bufs[k] = t
        p, mem, keep = self._input(cameras, "cameras")
        ptr = lambda k: C.c_void_p(bufs[k].data_ptr()) if k in bufs else None
        self._stream()
        check(self._lib.ngb_render_into(self._h, p, float(fov), int(samples_per_pixel), outputs, int(frame), mem,
                                        ptr("rgb"), ptr("depth"), ptr("normals"), ptr("object_ids")), self._h)
        self._keep = keep
        if zero_copy:
            return dict(bufs)
        host = {k: v.cpu().numpy() for k, v in bufs.items()}
        self.synchronize()  # reports a device-side error of this render
        return host

    def _render_host(self, cameras, fov, spp, rgb, depth, normals, object_ids, frame, out):
        views, h, w = self.view_count, self.rows[1], self.width
        _require_count(cameras, views * 12, "cameras", f"{views} cameras of 3 x 4 numbers (camera-to-world)")
        if _is_cuda_tensor(cameras):
            raise ValueError("render(out=...) copies to host memory and takes cameras in host memory")
        want = {"rgb": ((views, h, w, 3), np.uint8, rgb), "depth": ((views, h, w), np.float32, depth),
                "normals": ((views, h, w, 3), np.float32, normals), "object_ids": ((views, h, w), np.int32, object_ids)}
        ptrs = {}
        for k, (shape, dtype, on) in want.items():
            if not on:
                ptrs[k] = None
                continue
            a = out.get(k)
            if a is None or a.shape != shape or a.dtype != dtype or not a.flags.c_contiguous:
                raise ValueError(f"out['{k}'] must be a C-contiguous {np.dtype(dtype).name} array of shape {shape}")
            ptrs[k] = a.ctypes.data_as(C.c_void_p)
        outputs = ((_abi.OUTPUT_RGB if rgb else 0) | (_abi.OUTPUT_DEPTH if depth else 0) |
                   (_abi.OUTPUT_NORMAL if normals else 0) | (_abi.OUTPUT_OBJECT_ID if object_ids else 0))
        cams = np.ascontiguousarray(cameras, np.float32)
        self._stream()
        check(self._lib.ngb_render_host(self._h, cams.ctypes.data_as(C.c_void_p), float(fov), int(spp), outputs,
                                        int(frame), ptrs["rgb"], ptrs["depth"], ptrs["normals"], ptrs["object_ids"]),
              self._h)
        return {k: out[k] for k, v in ptrs.items() if v is not None}

    def cast_rays(self, origins, directions, max_distance=math.inf):
        """Rays in every world: (world_count, rays_per_world, 3) origins and directions. Returns distance
        (W, R), normal (W, R, 3) and object_id (W, R); CUDA tensors in give CUDA tensors out."""
        torch = _torch()
        worlds = self.world_count
        if _count(origins) % (3 * worlds) != 0:
            raise ValueError(f"origins must hold 3 floats for each ray of each of the {worlds} worlds: "
                             f"(world_count, rays_per_world, 3)")
        _require_count(directions, _count(origins), "directions", "the same as origins")
        rpw = _count(origins) // (3 * worlds)
        po, mo, ko = self._input(origins, "origins")
        pd, md, kd = self._input(directions, "directions")
        if mo != md:
            raise ValueError("origins and directions must be on the same device")
        dev = f"cuda:{self._device}"
        out = {"distance": torch.empty((worlds, rpw), dtype=torch.float32, device=dev),
               "normal": torch.empty((worlds, rpw, 3), dtype=torch.float32, device=dev),
               "object_id": torch.empty((worlds, rpw), dtype=torch.int32, device=dev)}
        ptr = lambda k: C.c_void_p(out[k].data_ptr()) if out[k].numel() else C.c_void_p(1)
        self._stream()
        check(self._lib.ngb_cast_rays_into(self._h, po, pd, rpw, float(max_distance), mo, ptr("distance"),
                                           ptr("normal"), ptr("object_id")), self._h)
        self._keep = (ko, kd)
        if mo == _abi.MEMORY_DEVICE:
            return out
        host = {k: v.cpu().numpy() for k, v in out.items()}
        self.synchronize()
        return host

    # ------------------------------------------------------------------------------------------- settings --

    def set_environment(self, environment: Environment):
        e = environment.to_abi()
        check(self._lib.ngb_set_environment(self._h, C.byref(e)), self._h)

    def set_lights(self, lights):
        """Replaces the lights (at most MAX_LIGHTS), checked as the constructor checks them."""
        lig = lights_abi(list(lights))
        check(self._lib.ngb_set_lights(self._h, lig, len(lights)), self._h)

    @property
    def ambient(self) -> float:
        return float(self._lib.ngb_ambient(self._h))

    @ambient.setter
    def ambient(self, value):
        check(self._lib.ngb_set_ambient(self._h, float(value)), self._h)

    @property
    def width(self) -> int:
        return int(self._lib.ngb_width(self._h))

    @property
    def height(self) -> int:
        return int(self._lib.ngb_height(self._h))

    @property
    def pixel_count(self) -> int:
        """Pixels of one output image of every view: views x rows drawn x width (uneven worlds: their sum)."""
        return int(self._lib.ngb_pixel_count(self._h))

    @property
    def rows(self) -> tuple:
        """(first, count): the image rows every render draws (set_rows); (0, height) for the whole image."""
        first, count = C.c_int32(0), C.c_int32(0)
        check(self._lib.ngb_rows(self._h, C.byref(first), C.byref(count)), self._h)
        return int(first.value), int(count.value)

    def set_rows(self, first=0, count=None):
        """Later renders draw image rows [first, first + count) of every view (count None: to the last row;
        set_rows() is the whole image again). Every pixel is the whole image's (the same rays and random
        streams); the outputs, hit records and the adjoint's per-pixel inputs hold (views, count, width). For
        splitting one large picture across GPUs by rows (sharding.ShardedFrame)."""
        if count is None:
            count = self.height - int(first)
        check(self._lib.ngb_set_rows(self._h, int(first), int(count)), self._h)

    @property
    def world_count(self) -> int:
        return int(self._lib.ngb_world_count(self._h))

    @property
    def cameras_per_world(self) -> int:
        return int(self._lib.ngb_cameras_per_world(self._h))

    @property
    def view_count(self) -> int:
        return int(self._lib.ngb_view_count(self._h))

    @property
    def instances_per_world(self) -> int:
        return int(self._lib.ngb_instances_per_world(self._h))

    @property
    def device(self) -> str:
        return "cuda"

    @property
    def last_kernel_ms(self) -> float:
        return float(self._lib.ngb_last_kernel_ms(self._h))

    @property
    def last_stage_ms(self) -> list:
        """The last render's GPU ms by kernel: [camera rays, shading, shadow rays] for the tile kernels, else
        [whole launch]."""
        ms = (C.c_float * 4)()
        n = C.c_int32(0)
        check(self._lib.ngb_last_stage_ms(self._h, ms, 4, C.byref(n)), self._h)
        return [float(ms[i]) for i in range(n.value)]

    def synchronize(self, timeout=_TIMEOUT_S):
        """Waits for the queued work (at most timeout seconds) and raises CudaError if a kernel reported an error."""
        check(self._lib.ngb_synchronize(self._h, float(timeout)), self._h)

    # ----------------------------------------------------------------------------------------- inspection --

    def set_tuning(self, kernel=0, threads_per_block=128, refill_lanes=28, registers=72, leaf_batch=16):
        """kernel: 0 automatic (the tile kernels where they apply), 1 the per-pixel kernel, 2 the persistent kernel
        (where it applies: one sample per pixel, at most one light, no reflective material), 3 the tile kernels
        (where the persistent kernel applies: per-tile candidate lists for worlds of at most 256 instances, a
        warp-packet walk of the world tree above). Ray queries keep a shape of their own unless kernel 2 is set. With kernel 3, threads_per_block and registers set the tile
        kernel's shape; otherwise they, refill_lanes and leaf_batch set the persistent kernel's (see
        ngb_set_tuning)."""
        check(self._lib.ngb_set_tuning(self._h, int(kernel), int(threads_per_block), int(refill_lanes), int(registers),
                                       int(leaf_batch)), self._h)

    def set_tile_shape(self, tiles_per_fetch=1, paired=True):
        """The tile kernels' work shape: tiles of 32 rays a warp takes per fetch (1 to 8), and whether a pixel's
        picture and centre rays share a 4 x 4 tile (paired) or run as 8 x 4 tiles of one kind. Same images."""
        check(self._lib.ngb_set_tile_shape(self._h, int(tiles_per_fetch), 1 if paired else 0), self._h)

    def set_ray_kernel(self, kernel=0):
        """Which kernel answers cast_rays: 0 automatic, 1 one thread per ray, 2 persistent (lane refill), 3 warp
        packets (32 consecutive rays per warp walking the world tree together). Same hits."""
        check(self._lib.ngb_set_ray_kernel(self._h, int(kernel)), self._h)

    def set_build(self, mode=0):
        """Instance-tree build: 0 automatic (per-world groups up to 1024 instances per world, else global),
        1 per-world, 2 global. Both make the same tree."""
        check(self._lib.ngb_set_build(self._h, int(mode)), self._h)

    def record_hits(self, on=True, into=None):
        """Later renders that ask for depth, normals or IDs also record each centre ray's hit. into: the
        caller's CUDA tensors (instance int32, triangle int32, u float32, v float32; each (views, H, W),
        contiguous) to write them to instead of the renderer's own buffers (no copy_hits needed); they must
        stay alive while renders may write them, until the next record_hits call."""
        if into is None:
            check(self._lib.ngb_record_hits(self._h, 1 if on else 0), self._h)
            return
        torch = _torch()
        shape = (self.view_count, self.rows[1], self.width)
        for t, dt in zip(into, (torch.int32, torch.int32, torch.float32, torch.float32)):
            if (not _is_cuda_tensor(t) or tuple(t.shape) != shape or t.dtype != dt or not t.is_contiguous() or
                    t.device.index != self._device):
                raise ValueError(f"record_hits(into=...) takes four contiguous CUDA tensors of shape {shape}: "
                                 "instance and triangle int32, u and v float32")
        check(self._lib.ngb_record_hits_into(self._h, *[C.c_void_p(t.data_ptr()) for t in into]), self._h)

    def inspect_tlas(self) -> dict:
        """The last tree build: keys (instance order), sorted ids, nodes (8 words), roots, matrices."""
        n = self.world_count * self.instances_per_world
        keys = np.zeros(n, np.uint64)
        ids = np.zeros(n, np.int32)
        nodes = np.zeros((max(2 * n - 1, 0), 8), np.int32)
        roots = np.zeros(self.world_count, np.int32)
        mats = np.zeros((n, 12), np.float32)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(self._lib.ngb_inspect_tlas(self._h, vp(keys), vp(ids), vp(nodes), vp(roots), vp(mats)), self._h)
        return {"keys": keys, "sorted_ids": ids, "nodes": nodes, "roots": roots, "matrices": mats}

    def copy_hits(self, instance, triangle, u, v):
        """Copies the last render's hit records into CUDA tensors of (views, height, width): int32 instance and
        triangle, float32 barycentrics (see ngb_copy_hits)."""
        ptr = lambda t: C.c_void_p(t.data_ptr())
        self._stream()
        check(self._lib.ngb_copy_hits(self._h, ptr(instance), ptr(triangle), ptr(u), ptr(v)), self._h)

    def depth_normal_adjoint(self, matrices, cameras, fov, hits, depth, grad_depth, grad_normal, grad_matrices,
                             grad_cameras):
        """Adds the gradients of the depth and normal images with respect to the instance matrices and the
        cameras into grad_matrices and grad_cameras (see ngb_depth_normal_adjoint). CUDA tensors throughout;
        hits = (instance, triangle, u, v) from copy_hits; grad_normal may be None."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(None)
        self._stream()
        check(self._lib.ngb_depth_normal_adjoint(self._h, ptr(matrices), ptr(cameras), float(fov), *map(ptr, hits),
                                                 ptr(depth), ptr(grad_depth), ptr(grad_normal), ptr(grad_matrices),
                                                 ptr(grad_cameras)), self._h)

    def inspect_hits(self) -> dict:
        shape = (self.view_count, self.rows[1], self.width)
        inst, tri = np.zeros(shape, np.int32), np.zeros(shape, np.int32)
        u, v = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(self._lib.ngb_inspect_hits(self._h, vp(inst), vp(tri), vp(u), vp(v)), self._h)
        return {"hit_instance": inst, "hit_triangle": tri, "hit_u": u, "hit_v": v}


class UnevenBatchRenderer(BatchRenderer):
    """Worlds of uneven instance counts and image sizes in one renderer (ngb_create_uneven).

    worlds: a list of (width, height, instances), one camera per world; every world may hold its own list of
    0 to 256 instances of the shared meshes. Matrices for set_instance_transforms are every world's instances,
    world after world: (total_instances, 3, 4). render takes (world_count, 3, 4) cameras and returns the images
    packed world after world: 'rgb' (pixels, 3), 'depth' (pixels,), 'normals' (pixels, 3), 'object_ids'
    (pixels,); image(out, w) views world w's image as (height, width[, 3]). One sample per pixel, at most one
    light and no reflective material.
    """

    def __init__(self, worlds, spheres=(), lights=(), floor=None, meshes=(), device="auto"):
        self._device = _parse_device(device)
        flat = [inst for _, _, insts in worlds for inst in insts]
        self._desc = SceneDesc(1, 1, 1, 1, spheres, lights, floor if floor is not None else Plane(), meshes, flat,
                               self._device)
        self._sizes = [(int(w), int(h)) for w, h, _ in worlds]
        self._counts = [len(insts) for _, _, insts in worlds]
        arr = (_abi.UnevenWorldC * len(worlds))(*[_abi.UnevenWorldC(w, h, c) for (w, h), c in zip(self._sizes,
                                                                                                  self._counts)])
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.ngb_create_uneven(C.byref(self._desc.c), arr, len(worlds), C.byref(h)), None)
        self._h = h
        check(self._lib.ngb_set_sync(self._h, 0, _TIMEOUT_S), self._h)
        self._out = {}
        self._rays = {}
        self.pixel_first = np.concatenate([[0], np.cumsum([w * hh for w, hh in self._sizes])]).astype(np.int64)
        self.instance_first = np.concatenate([[0], np.cumsum(self._counts)]).astype(np.int64)

    @property
    def instance_count(self) -> int:
        return int(self.instance_first[-1])

    def set_instance_transforms(self, matrices):
        """Every world's instance matrices, world after world: (total_instances, 3, 4) float32."""
        _require_count(matrices, self.instance_count * 12, "matrices", "(total_instances, 3, 4)")
        p, mem, keep = self._input(matrices, "matrices")
        self._stream()
        check(self._lib.ngb_set_instance_transforms(self._h, p, mem), self._h)
        self._keep = keep
        if mem == _abi.MEMORY_HOST:
            self.synchronize()

    def bind_bodies(self, *args, **kwargs):
        raise ValueError("worlds of uneven sizes take instance matrices (set_instance_transforms), not body poses")

    def bind_geoms(self, *args, **kwargs):
        raise ValueError("worlds of uneven sizes take instance matrices (set_instance_transforms), not geom poses")

    def render(self, cameras, fov=1.0, samples_per_pixel=1, *, rgb=True, depth=False, normals=False,
               object_ids=False, frame=0, zero_copy=False):
        torch = _torch()
        P, worlds = self.pixel_count, len(self._sizes)
        _require_count(cameras, worlds * 12, "cameras", f"{worlds} cameras of 3 x 4 numbers (camera-to-world)")
        if not zero_copy and _is_cuda_tensor(cameras):
            raise ValueError("cameras on the GPU need zero_copy=True: the results then stay on the GPU too")
        outputs = ((_abi.OUTPUT_RGB if rgb else 0) | (_abi.OUTPUT_DEPTH if depth else 0) |
                   (_abi.OUTPUT_NORMAL if normals else 0) | (_abi.OUTPUT_OBJECT_ID if object_ids else 0))
        bufs = {}
        if rgb:
            bufs["rgb"] = self._buffer("rgb", (P, 3), torch.uint8)
        if depth:
            bufs["depth"] = self._buffer("depth", (P,), torch.float32)
        if normals:
            bufs["normals"] = self._buffer("normals", (P, 3), torch.float32)
        if object_ids:
            bufs["object_ids"] = self._buffer("object_ids", (P,), torch.int32)
        p, mem, keep = self._input(cameras, "cameras")
        ptr = lambda k: C.c_void_p(bufs[k].data_ptr()) if k in bufs else None
        self._stream()
        check(self._lib.ngb_render_into(self._h, p, float(fov), int(samples_per_pixel), outputs, int(frame), mem,
                                        ptr("rgb"), ptr("depth"), ptr("normals"), ptr("object_ids")), self._h)
        self._keep = keep
        if zero_copy:
            return dict(bufs)
        host = {k: v.cpu().numpy() for k, v in bufs.items()}
        self.synchronize()
        return host

    def image(self, packed, w):
        """World w's image out of a packed output: (height, width) or (height, width, 3)."""
        a, b = int(self.pixel_first[w]), int(self.pixel_first[w + 1])
        width, height = self._sizes[w]
        x = packed[a:b]
        return x.reshape((height, width) + tuple(x.shape[1:]))


class _DeviceArray:
    """A device array the renderer owns, as __cuda_array_interface__ describes it, for a zero-copy torch view."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _device_view(ptr, shape, dtype, device):
    torch = _torch()
    typestr = {torch.uint8: "|u1", torch.float32: "<f4", torch.int32: "<i4"}[dtype]
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr), device=f"cuda:{device}")


def _camera_c(camera) -> _abi.CameraC:
    """An ngb_camera from a scene.Camera (or anything with its six fields)."""
    v = lambda t: _abi.Vec3(float(t[0]), float(t[1]), float(t[2]))
    return _abi.CameraC(v(camera.position), v(camera.right), v(camera.up), v(camera.forward), float(camera.fov_scale),
                        float(camera.aspect))


class Renderer:
    """The reference's single-view Renderer (include/neraulgraphics/renderer.h:135-277, python/bindings.cpp:801-943):
    one scene seen by one camera, over a one-world BatchRenderer and the C ABI's view calls.

    render() traces one frame and averages it with the frames before it (frame 0 starts afresh); render_frame()
    returns the images asked for; cast_rays() answers ray queries; set_instance_transforms() moves the instances.
    Cameras are scene.Camera objects (make_camera), used as given."""

    def __init__(self, width, height, spheres=(), lights=(), floor=None, meshes=(), instances=(), device="auto"):
        self._batch = BatchRenderer(width, height, 1, 1, spheres, lights, floor, meshes, instances, device=device)
        self._lib = self._batch._lib
        self._h = self._batch._h

    def __repr__(self):
        return f"Renderer({self.width}x{self.height}, {self.instance_count} instances, {self.device})"

    def set_instance_transforms(self, transforms):
        """Move the instances: (N, 3, 4) matrices (host arrays, checked; CUDA tensors, used where they are), or a
        list of Transform objects."""
        if isinstance(transforms, (list, tuple)) and transforms and hasattr(transforms[0], "matrix"):
            transforms = np.stack([np.asarray(t.matrix, np.float32) for t in transforms])
        self._batch.set_instance_transforms(transforms)

    def render(self, camera, frame=0, samples_per_frame=1):
        """One frame, averaged with the frames before it: a (height, width, 3) uint8 RGB array (the 0xAARRGGBB
        pixels of Renderer::render, unpacked)."""
        argb = self.render_argb(camera, frame, samples_per_frame)
        out = np.empty(argb.shape + (3,), np.uint8)
        out[..., 0] = (argb >> 16) & 0xFF
        out[..., 1] = (argb >> 8) & 0xFF
        out[..., 2] = argb & 0xFF
        return out

    def render_argb(self, camera, frame=0, samples_per_frame=1):
        """The same picture as (height, width) uint32 0xAARRGGBB pixels, as Renderer::render returns them."""
        h, w = self._batch.rows[1], self.width
        argb = np.empty((h, w), np.uint32)
        cam = _camera_c(camera)
        self._batch._stream()
        check(self._lib.ngb_render_view(self._h, C.byref(cam), int(frame), int(samples_per_frame),
                                        argb.ctypes.data_as(C.c_void_p)), self._h)
        return argb

    def render_frame(self, camera, frame=0, samples_per_frame=1, *, rgb=True, depth=False, normals=False,
                     object_ids=False, zero_copy=False):
        """The images asked for: 'rgb' (H, W, 3) uint8 (the running average's bytes; it advances the average as
        render() does), 'depth' (H, W) float32, 'normals' (H, W, 3) float32, 'object_ids' (H, W) int32. Copies by
        default; with zero_copy=True, CUDA tensors aliasing the renderer's own buffers, queued on PyTorch's current
        stream and overwritten by the next render."""
        torch = _torch()
        outputs = ((_abi.OUTPUT_RGB if rgb else 0) | (_abi.OUTPUT_DEPTH if depth else 0) |
                   (_abi.OUTPUT_NORMAL if normals else 0) | (_abi.OUTPUT_OBJECT_ID if object_ids else 0))
        cam = _camera_c(camera)
        f = _abi.BatchFrameC()
        self._batch._stream()
        check(self._lib.ngb_render_view_frame(self._h, C.byref(cam), int(frame), int(samples_per_frame), outputs,
                                              C.byref(f)), self._h)
        h, w = f.height, f.width
        images = {"rgb": (f.rgb, (h, w, 3), torch.uint8), "depth": (f.depth, (h, w), torch.float32),
                  "normals": (f.normal, (h, w, 3), torch.float32), "object_ids": (f.object_id, (h, w), torch.int32)}
        views = {k: _device_view(ptr, shape, dtype, self._batch._device) for k, (ptr, shape, dtype) in images.items()
                 if ptr}
        if zero_copy:
            return views
        host = {k: v.cpu().numpy() for k, v in views.items()}
        self._batch.synchronize()
        return host

    def cast_rays(self, origins, directions, max_distance=math.inf):
        """Rays into the scene: (N, 3) origins and directions (directions need not be unit length). Returns
        'distance' (N,), 'normal' (N, 3) and 'object_id' (N,); CUDA tensors in give CUDA tensors out."""
        if _count(origins) != _count(directions):
            raise ValueError("origins and directions must have the same number of rays")
        hits = self._batch.cast_rays(origins, directions, max_distance)
        return {k: v[0] for k, v in hits.items()}

    def set_environment(self, environment: Environment):
        self._batch.set_environment(environment)

    def set_lights(self, lights):
        """Replaces the lights: a flashlight that follows a camera, a lamp that flickers."""
        self._batch.set_lights(lights)

    @property
    def ambient(self) -> float:
        return self._batch.ambient

    @ambient.setter
    def ambient(self, value):
        self._batch.ambient = value

    @property
    def instance_count(self) -> int:
        return self._batch.instances_per_world

    @property
    def width(self) -> int:
        return self._batch.width

    @property
    def height(self) -> int:
        return self._batch.height

    @property
    def device(self) -> str:
        return self._batch.device

    @property
    def last_kernel_ms(self) -> float:
        return self._batch.last_kernel_ms

    def set_tuning(self, *args, **kwargs):
        self._batch.set_tuning(*args, **kwargs)

    def synchronize(self, timeout=_TIMEOUT_S):
        self._batch.synchronize(timeout)
