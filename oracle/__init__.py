"""TEST INFRASTRUCTURE ONLY: the checkers the parity tests compare the product against.

- `Oracle`: the C restatement of the reference's path (oracle.c, built into liboracle.so).
- `Reference`: the reference implementation itself (neraulgraphics 0.5.0, its CPU backend, or its CUDA
  backend when oracle/_ref/libngref_cuda.so was built), compiled from its own sources into oracle/_ref/
  by oracle/Makefile, driven through the small C ABI of ref_harness.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package, and only as the
checker. The product never imports it.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from neraulgraphics_b200 import _abi
from neraulgraphics_b200.scene import Mesh, SceneDesc

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libngref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libngref_cuda.so")
REF_TLAS_SO = os.path.join(HERE, "_ref", "libngref_tlas.so")
REF_NGB_SO = os.path.join(HERE, "_ref", "libngref_ngb.so")

TIE_AOV_INSTANCE = 1
TIE_AOV_TRIANGLE = 2
TIE_RGB_INSTANCE = 4

_f32p = C.POINTER(C.c_float)


def _p(a, ctype=C.c_float):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


_oracle_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} is not built: run `make -C oracle`")
        lib = C.CDLL(ORACLE_SO)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(_abi.SceneC), C.c_char_p, C.c_int]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_set_instance_transforms.argtypes = [C.c_void_p, _f32p]
        lib.orc_bind_bodies.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int32), _f32p, _f32p]
        lib.orc_set_body_poses.argtypes = [C.c_void_p, _f32p]
        lib.orc_set_ambient.argtypes = [C.c_void_p, C.c_float]
        lib.orc_set_environment.argtypes = [C.c_void_p, C.POINTER(_abi.EnvironmentC)]
        lib.orc_render.argtypes = [C.c_void_p, _f32p, C.c_float, C.c_int, C.c_uint, C.c_int,
                                   C.POINTER(C.c_uint8), _f32p, _f32p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int32), _f32p, _f32p, C.POINTER(C.c_uint8), C.c_int]
        lib.orc_cast_rays.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int, C.c_float, _f32p, _f32p, C.POINTER(C.c_int32)]
        lib.orc_tlas.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32), _f32p]
        lib.orc_blas.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int32), _f32p,
                                 C.POINTER(C.c_int32), _f32p, C.POINTER(C.c_int32)]
        lib.orc_traversal_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.orc_compose.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32), _f32p, _f32p, _f32p, _f32p]
        lib.orc_render_view.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_uint, C.c_int, _f32p, C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint8), _f32p, _f32p, C.POINTER(C.c_int32),
                                        C.POINTER(C.c_uint8), C.c_int]
        _oracle_lib = lib
    return _oracle_lib


def _images(views, h, w, outputs):
    out = {}
    if outputs & _abi.OUTPUT_RGB:
        out["rgb"] = np.zeros((views, h, w, 3), np.uint8)
    if outputs & _abi.OUTPUT_DEPTH:
        out["depth"] = np.zeros((views, h, w), np.float32)
    if outputs & _abi.OUTPUT_NORMAL:
        out["normals"] = np.zeros((views, h, w, 3), np.float32)
    if outputs & _abi.OUTPUT_OBJECT_ID:
        out["object_ids"] = np.zeros((views, h, w), np.int32)
    return out


def outputs_mask(rgb=True, depth=False, normals=False, object_ids=False) -> int:
    return ((_abi.OUTPUT_RGB if rgb else 0) | (_abi.OUTPUT_DEPTH if depth else 0) |
            (_abi.OUTPUT_NORMAL if normals else 0) | (_abi.OUTPUT_OBJECT_ID if object_ids else 0))


class Oracle:
    """The C restatement of the reference's path over one scene."""

    def __init__(self, desc: SceneDesc):
        self.lib = oracle_lib()
        self.desc = desc
        err = C.create_string_buffer(512)
        self.h = self.lib.orc_create(C.byref(desc.c), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_instance_transforms(self, matrices):
        m = np.ascontiguousarray(matrices, np.float32)
        self.lib.orc_set_instance_transforms(self.h, _p(m))

    def bind_bodies(self, body_of_instance, local_pose, scale, bodies_per_world):
        b = np.ascontiguousarray(body_of_instance, np.int32)
        lp = np.ascontiguousarray(local_pose, np.float32)
        sc = np.ascontiguousarray(scale, np.float32)
        self.lib.orc_bind_bodies(self.h, int(bodies_per_world), _p(b, C.c_int32), _p(lp), _p(sc))

    def set_body_poses(self, poses):
        p = np.ascontiguousarray(poses, np.float32)
        if self.lib.orc_set_body_poses(self.h, _p(p)) != 0:
            raise ValueError("set_body_poses needs bind_bodies to be called first")

    def set_ambient(self, a):
        self.lib.orc_set_ambient(self.h, float(a))

    def set_environment(self, env):
        e = env.to_abi()
        self.lib.orc_set_environment(self.h, C.byref(e))

    def render(self, cameras, fov=1.0, samples_per_pixel=1, *, rgb=True, depth=False, normals=False,
               object_ids=False, frame=0, hits=False, ties=False, threads=0):
        d = self.desc
        cams = np.ascontiguousarray(cameras, np.float32)
        outputs = outputs_mask(rgb, depth, normals, object_ids)
        out = _images(d.view_count, d.height, d.width, outputs)
        shape = (d.view_count, d.height, d.width)
        hi = ht = hu = hv = tf = None
        if hits:
            hi, ht = np.zeros(shape, np.int32), np.zeros(shape, np.int32)
            hu, hv = np.zeros(shape, np.float32), np.zeros(shape, np.float32)
        if ties:
            tf = np.zeros(shape, np.uint8)
        self.lib.orc_render(self.h, _p(cams), float(fov), int(samples_per_pixel), outputs, int(frame),
                            _p(out.get("rgb"), C.c_uint8), _p(out.get("depth")), _p(out.get("normals")),
                            _p(out.get("object_ids"), C.c_int32), _p(hi, C.c_int32), _p(ht, C.c_int32), _p(hu),
                            _p(hv), _p(tf, C.c_uint8), int(threads))
        if hits:
            out.update(hit_instance=hi, hit_triangle=ht, hit_u=hu, hit_v=hv)
        if ties:
            out["ties"] = tf
        return out

    def render_view(self, camera, frame=0, samples_per_frame=1, *, rgb=True, depth=False, normals=False,
                    object_ids=False, ties=False, threads=0):
        """The single-view Renderer's render / render_frame on a scene of one world and one camera (a
        scene.Camera, used as given): the running average's 'argb' (H, W) uint32 and 'rgb' bytes, and the other
        images asked for. The average carries over between calls on this oracle; frame 0 starts it."""
        d = self.desc
        cam = np.float32(list(camera.position) + list(camera.right) + list(camera.up) + list(camera.forward) +
                         [camera.fov_scale, camera.aspect])
        if getattr(self, "_accum", None) is None:
            self._accum = np.zeros((d.height, d.width, 4), np.float32)
        outputs = outputs_mask(rgb, depth, normals, object_ids)
        out = {k: v[0] for k, v in _images(1, d.height, d.width, outputs).items()}
        argb = np.zeros((d.height, d.width), np.uint32) if rgb else None
        tf = np.zeros((d.height, d.width), np.uint8) if ties else None
        self.lib.orc_render_view(self.h, _p(cam), int(samples_per_frame), outputs, int(frame),
                                 _p(self._accum) if rgb else None, _p(argb, C.c_uint32), _p(out.get("rgb"), C.c_uint8),
                                 _p(out.get("depth")), _p(out.get("normals")), _p(out.get("object_ids"), C.c_int32),
                                 _p(tf, C.c_uint8), int(threads))
        if rgb:
            out["argb"] = argb
        if ties:
            out["ties"] = tf
        return out

    def cast_rays(self, origins, directions, max_distance=np.inf):
        o = np.ascontiguousarray(origins, np.float32)
        dd = np.ascontiguousarray(directions, np.float32)
        worlds = self.desc.world_count
        rpw = o.size // (3 * worlds)
        dist = np.zeros((worlds, rpw), np.float32)
        nrm = np.zeros((worlds, rpw, 3), np.float32)
        ids = np.zeros((worlds, rpw), np.int32)
        self.lib.orc_cast_rays(self.h, _p(o), _p(dd), rpw, float(max_distance), _p(dist), _p(nrm), _p(ids, C.c_int32))
        return {"distance": dist, "normal": nrm, "object_id": ids}

    def tlas(self):
        n = self.desc.world_count * self.desc.per_world
        keys = np.zeros(n, np.uint64)
        ids = np.zeros(n, np.int32)
        nodes = np.zeros((max(2 * n - 1, 0), 8), np.int32)
        roots = np.zeros(self.desc.world_count, np.int32)
        mats = np.zeros((n, 12), np.float32)
        self.lib.orc_tlas(self.h, _p(keys, C.c_uint64), _p(ids, C.c_int32), _p(nodes, C.c_int32), _p(roots, C.c_int32),
                          _p(mats))
        return {"keys": keys, "sorted_ids": ids, "nodes": nodes, "roots": roots, "matrices": mats}

    def blas(self):
        nn, nt = C.c_int(), C.c_int()
        self.lib.orc_blas(self.h, C.byref(nn), C.byref(nt), None, None, None, None, None)
        nodes = np.zeros((nn.value, 8), np.int32)
        tris = np.zeros((nt.value, 12), np.float32)
        m = len(self.desc.meshes)
        roots = np.zeros(m, np.int32)
        bounds = np.zeros((m, 6), np.float32)
        tidx = np.zeros(nt.value, np.int32)
        self.lib.orc_blas(self.h, C.byref(nn), C.byref(nt), _p(nodes, C.c_int32), _p(tris), _p(roots, C.c_int32),
                          _p(bounds), _p(tidx, C.c_int32))
        return {"nodes": nodes, "triangles": tris, "roots": roots, "bounds": bounds, "triangle_index": tidx}

    def traversal_bytes(self):
        b, r = C.c_double(), C.c_double()
        self.lib.orc_traversal_bytes(self.h, C.byref(b), C.byref(r))
        return b.value, r.value


def compose(worlds, per_world, bodies_per_world, body_of_instance, local_pose, scale, poses):
    """The single-precision compose of the reference's GPU kernel, restated (oracle.c:orc_compose)."""
    lib = oracle_lib()
    b = np.ascontiguousarray(body_of_instance, np.int32)
    lp = np.ascontiguousarray(local_pose, np.float32)
    sc = np.ascontiguousarray(scale, np.float32)
    p = np.ascontiguousarray(poses, np.float32)
    out = np.zeros((worlds, per_world, 3, 4), np.float32)
    lib.orc_compose(worlds, per_world, bodies_per_world, _p(b, C.c_int32), _p(lp), _p(sc), _p(p), _p(out))
    return out


def geom_matrices(geom_xpos, geom_xmat, geom_of_instance, scale):
    """Instance matrices from MuJoCo geom poses, [R * diag(scale) | p] per instance in float32: the products
    of MJWarpBatchRenderer's compose kernel (python/neraulgraphics/mujoco.py:291-302), one rounding each.
    geom_xpos (worlds, geoms, 3), geom_xmat (worlds, geoms, 3, 3) -> (worlds, instances, 3, 4)."""
    g = np.asarray(geom_of_instance, np.int64)
    xpos = np.asarray(geom_xpos, np.float32)
    xmat = np.asarray(geom_xmat, np.float32).reshape(xpos.shape[0], xpos.shape[1], 3, 3)
    s = np.asarray(scale, np.float32).reshape(-1, 3)
    out = np.empty((xpos.shape[0], len(g), 3, 4), np.float32)
    out[..., :3] = xmat[:, g] * s[None, :, None, :]
    out[..., 3] = xpos[:, g]
    return out


# ---------------------------------------------------------------------------- the reference itself --

_ref_libs: dict = {}


def reference_available(cuda=False, ngb=False) -> bool:
    return os.path.exists(REF_NGB_SO if ngb else REF_CUDA_SO if cuda else REF_SO)


def ref_lib(cuda=False, ngb=False):
    """The reference's library: its CPU backend, its CUDA backend (cuda), or its Device::Cuda drawing through this
    library by oracle/ngb_backend.cpp (ngb)."""
    path = REF_NGB_SO if ngb else REF_CUDA_SO if cuda else REF_SO
    if path not in _ref_libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built: run `make -C oracle ref` where the reference's sources are")
        lib = C.CDLL(path)
        lib.ngref_last_error.restype = C.c_char_p
        lib.ngref_set_threads.argtypes = [C.c_int]
        lib.ngref_create.argtypes = [C.POINTER(_abi.SceneC), C.c_int, C.POINTER(C.c_void_p)]
        lib.ngref_destroy.argtypes = [C.c_void_p]
        lib.ngref_set_instance_transforms.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.ngref_bind_bodies.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int32), _f32p, _f32p, C.c_int]
        lib.ngref_set_body_poses.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.ngref_set_ambient.argtypes = [C.c_void_p, C.c_float]
        lib.ngref_render_host.argtypes = [C.c_void_p, _f32p, C.c_float, C.c_int, C.c_uint, C.c_int,
                                          C.POINTER(C.c_uint8), _f32p, _f32p, C.POINTER(C.c_int32)]
        lib.ngref_render.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_uint, C.c_int, C.c_int,
                                     C.POINTER(_abi.BatchFrameC)]
        lib.ngref_cast_rays_host.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int, C.c_int, C.c_float, _f32p, _f32p,
                                             C.POINTER(C.c_int32)]
        if hasattr(lib, "ngref_cast_rays_device"):
            lib.ngref_cast_rays_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float]
        lib.ngref_last_kernel_ms.restype = C.c_float
        lib.ngref_last_kernel_ms.argtypes = [C.c_void_p]
        lib.ngref_device.argtypes = [C.c_void_p]
        lib.ngref_build_meshes.argtypes = [C.POINTER(_abi.MeshC), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_int32), _f32p, C.POINTER(C.c_int32), _f32p]
        lib.ngref_body_poses_to_matrices.argtypes = [C.c_int, C.POINTER(C.c_int32), _f32p, _f32p, C.c_int, C.c_int,
                                                     _f32p, _f32p]
        lib.ngref_make_icosphere.argtypes = [C.c_float, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _f32p,
                                             C.POINTER(C.c_uint32)]
        lib.ngref_make_box.argtypes = [C.c_float, C.c_float, C.c_float, _f32p, C.POINTER(C.c_uint32)]
        lib.ngref_make_transform.argtypes = [_f32p, _f32p, C.c_float, _f32p]
        lib.ngref_camera_matrix.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_int, C.c_int, _f32p]
        lib.ngref_invert_affine.argtypes = [_f32p, _f32p]
        lib.ngref_transform_aabb.argtypes = [_f32p, _f32p, _f32p]
        _ref_libs[path] = lib
    return _ref_libs[path]


def _use_meshes(lib, desc):
    """The meshes ngb_backend.cpp hands the library (the reference's backend seam carries only their trees)."""
    lib.ngref_use_meshes.argtypes = [C.POINTER(_abi.MeshC), C.c_int]
    lib.ngref_use_meshes(desc.c.meshes, desc.c.mesh_count)


class ReferenceError_(ValueError):
    pass


def _ref_check(lib, status):
    if status != 0:
        msg = lib.ngref_last_error().decode()
        if status == 1:
            raise ValueError(msg)
        raise RuntimeError(msg)


class Reference:
    """neraulgraphics 0.5.0's own BatchRenderer (Device::Cpu, or Device::Cuda with cuda=True)."""

    def __init__(self, desc: SceneDesc, cuda=False, threads=None, ngb=False):
        self.lib = ref_lib(cuda, ngb)
        self.desc = desc
        if threads is not None:
            self.lib.ngref_set_threads(int(threads))
        if ngb:
            _use_meshes(self.lib, desc)
        h = C.c_void_p()
        _ref_check(self.lib, self.lib.ngref_create(C.byref(desc.c), 1 if (cuda or ngb) else 0, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ngref_destroy(self.h)
            self.h = None

    def set_instance_transforms(self, matrices, device=False):
        if device:
            _ref_check(self.lib, self.lib.ngref_set_instance_transforms(self.h, C.c_void_p(matrices), 1))
            return
        m = np.ascontiguousarray(matrices, np.float32)
        _ref_check(self.lib, self.lib.ngref_set_instance_transforms(self.h, m.ctypes.data_as(C.c_void_p), 0))

    def bind_bodies(self, body_of_instance, local_pose, scale, bodies_per_world):
        b = np.ascontiguousarray(body_of_instance, np.int32)
        lp = np.ascontiguousarray(local_pose, np.float32)
        sc = np.ascontiguousarray(scale, np.float32)
        _ref_check(self.lib, self.lib.ngref_bind_bodies(self.h, int(bodies_per_world), _p(b, C.c_int32), _p(lp), _p(sc),
                                                        len(b)))

    def set_body_poses(self, poses, device=False):
        if device:
            _ref_check(self.lib, self.lib.ngref_set_body_poses(self.h, C.c_void_p(poses), 1))
            return
        p = np.ascontiguousarray(poses, np.float32)
        _ref_check(self.lib, self.lib.ngref_set_body_poses(self.h, p.ctypes.data_as(C.c_void_p), 0))

    def set_ambient(self, a):
        _ref_check(self.lib, self.lib.ngref_set_ambient(self.h, float(a)))

    def render(self, cameras, fov=1.0, samples_per_pixel=1, *, rgb=True, depth=False, normals=False,
               object_ids=False, frame=0):
        d = self.desc
        cams = np.ascontiguousarray(cameras, np.float32)
        outputs = outputs_mask(rgb, depth, normals, object_ids)
        out = _images(d.view_count, d.height, d.width, outputs)
        _ref_check(self.lib, self.lib.ngref_render_host(self.h, _p(cams), float(fov), int(samples_per_pixel), outputs,
                                                        int(frame), _p(out.get("rgb"), C.c_uint8), _p(out.get("depth")),
                                                        _p(out.get("normals")), _p(out.get("object_ids"), C.c_int32)))
        return out

    def render_device(self, camera_ptr, fov, spp, outputs, frame=0):
        """Renders from device cameras and leaves the images on the device (Device::Cuda only)."""
        f = _abi.BatchFrameC()
        _ref_check(self.lib, self.lib.ngref_render(self.h, C.c_void_p(camera_ptr), float(fov), int(spp), int(outputs),
                                                   int(frame), 1, C.byref(f)))
        return f

    def cast_rays_device(self, origin_ptr, direction_ptr, rays_per_world, max_distance):
        """Rays already in device memory (CUDA reference only); the hits stay on the device."""
        _ref_check(self.lib, self.lib.ngref_cast_rays_device(self.h, C.c_void_p(origin_ptr), C.c_void_p(direction_ptr),
                                                             int(rays_per_world), float(max_distance)))

    def cast_rays(self, origins, directions, max_distance=np.inf):
        o = np.ascontiguousarray(origins, np.float32)
        dd = np.ascontiguousarray(directions, np.float32)
        worlds = self.desc.world_count
        rpw = o.size // (3 * worlds)
        dist = np.zeros((worlds, rpw), np.float32)
        nrm = np.zeros((worlds, rpw, 3), np.float32)
        ids = np.zeros((worlds, rpw), np.int32)
        _ref_check(self.lib, self.lib.ngref_cast_rays_host(self.h, _p(o), _p(dd), rpw, worlds, float(max_distance),
                                                           _p(dist), _p(nrm), _p(ids, C.c_int32)))
        return {"distance": dist, "normal": nrm, "object_id": ids}

    @property
    def last_kernel_ms(self) -> float:
        return float(self.lib.ngref_last_kernel_ms(self.h))


class ReferenceView:
    """neraulgraphics 0.5.0's own single-view Renderer (Device::Cpu, or Device::Cuda with cuda=True) on a scene
    of one world (desc.width x desc.height)."""

    def __init__(self, desc: SceneDesc, cuda=False, threads=None, ngb=False):
        self.lib = ref_lib(cuda, ngb)
        for name, args in (("ngref_view_create", [C.POINTER(_abi.SceneC), C.c_int, C.POINTER(C.c_void_p)]),
                           ("ngref_view_destroy", [C.c_void_p]), ("ngref_view_set_matrices", [C.c_void_p, _f32p]),
                           ("ngref_view_set_ambient", [C.c_void_p, C.c_float]),
                           ("ngref_view_render", [C.c_void_p, C.POINTER(_abi.CameraC), C.c_int, C.c_int,
                                                  C.POINTER(C.c_uint32)]),
                           ("ngref_view_render_frame", [C.c_void_p, C.POINTER(_abi.CameraC), C.c_int, C.c_int, C.c_uint,
                                                        C.POINTER(C.c_uint8), _f32p, _f32p, C.POINTER(C.c_int32)])):
            getattr(self.lib, name).argtypes = args
        self.desc = desc
        if threads is not None:
            self.lib.ngref_set_threads(int(threads))
        if ngb:
            _use_meshes(self.lib, desc)
        h = C.c_void_p()
        _ref_check(self.lib, self.lib.ngref_view_create(C.byref(desc.c), 1 if (cuda or ngb) else 0, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ngref_view_destroy(self.h)
            self.h = None

    @staticmethod
    def _camera(camera):
        v = lambda t: _abi.Vec3(float(t[0]), float(t[1]), float(t[2]))
        return _abi.CameraC(v(camera.position), v(camera.right), v(camera.up), v(camera.forward),
                            float(camera.fov_scale), float(camera.aspect))

    def set_instance_transforms(self, matrices):
        m = np.ascontiguousarray(matrices, np.float32)
        _ref_check(self.lib, self.lib.ngref_view_set_matrices(self.h, _p(m)))

    def set_ambient(self, a):
        _ref_check(self.lib, self.lib.ngref_view_set_ambient(self.h, float(a)))

    def render(self, camera, frame=0, samples_per_frame=1):
        """Renderer::render: (H, W) uint32 0xAARRGGBB."""
        out = np.zeros((self.desc.height, self.desc.width), np.uint32)
        cam = self._camera(camera)
        _ref_check(self.lib, self.lib.ngref_view_render(self.h, C.byref(cam), int(frame), int(samples_per_frame),
                                                        _p(out, C.c_uint32)))
        return out

    def render_frame(self, camera, frame=0, samples_per_frame=1, *, rgb=True, depth=False, normals=False,
                     object_ids=False):
        d = self.desc
        outputs = outputs_mask(rgb, depth, normals, object_ids)
        out = {k: v[0] for k, v in _images(1, d.height, d.width, outputs).items()}
        cam = self._camera(camera)
        _ref_check(self.lib, self.lib.ngref_view_render_frame(self.h, C.byref(cam), int(frame), int(samples_per_frame),
                                                              outputs, _p(out.get("rgb"), C.c_uint8),
                                                              _p(out.get("depth")), _p(out.get("normals")),
                                                              _p(out.get("object_ids"), C.c_int32)))
        return out


def ref_tlas_available() -> bool:
    return os.path.exists(REF_TLAS_SO)


def ref_tlas_cuda(worlds, per_world, local_bounds, matrices):
    """The reference's own GPU instance-tree build (src/cuda_tlas.cuh, compiled with its -use_fast_math flags into
    oracle/_ref/libngref_tlas.so by ref_tlas_cuda.cu) over these matrices: keys in instance order, sorted ids,
    nodes (2n - 1, 8 words) and roots, as ngb_inspect_tlas gives them. Needs a GPU."""
    if "tlas" not in _ref_libs:
        if not os.path.exists(REF_TLAS_SO):
            raise RuntimeError(f"{REF_TLAS_SO} is not built: run `make -C oracle ref-cuda` where the reference's sources are")
        lib = C.CDLL(REF_TLAS_SO)
        lib.ngref_tlas_last_error.restype = C.c_char_p
        lib.ngref_tlas_build.argtypes = [C.c_int, C.c_int, _f32p, _f32p, C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        _ref_libs["tlas"] = lib
    lib = _ref_libs["tlas"]
    n = worlds * per_world
    lb = np.ascontiguousarray(local_bounds, np.float32).reshape(per_world, 6)
    m = np.ascontiguousarray(matrices, np.float32).reshape(n, 12)
    keys = np.zeros(n, np.uint64)
    ids = np.zeros(n, np.int32)
    nodes = np.zeros((2 * n - 1, 8), np.int32)
    roots = np.zeros(worlds, np.int32)
    if lib.ngref_tlas_build(int(worlds), int(per_world), _p(lb), _p(m), _p(keys, C.c_uint64), _p(ids, C.c_int32),
                            _p(nodes, C.c_int32), _p(roots, C.c_int32)) != 0:
        raise RuntimeError(lib.ngref_tlas_last_error().decode())
    return {"keys": keys, "sorted_ids": ids, "nodes": nodes, "roots": roots}


def ref_build_meshes(meshes):
    """The reference's detail::build_meshes: nodes (8 words), packed triangles, roots, bounds."""
    lib = ref_lib()
    desc = SceneDesc(1, 1, 1, meshes=meshes)
    nn, nt = C.c_int(), C.c_int()
    _ref_check(lib, lib.ngref_build_meshes(desc.c.meshes, len(meshes), C.byref(nn), C.byref(nt), None, None, None, None))
    nodes = np.zeros((nn.value, 8), np.int32)
    tris = np.zeros((nt.value, 12), np.float32)
    roots = np.zeros(len(meshes), np.int32)
    bounds = np.zeros((len(meshes), 6), np.float32)
    _ref_check(lib, lib.ngref_build_meshes(desc.c.meshes, len(meshes), C.byref(nn), C.byref(nt), _p(nodes, C.c_int32),
                                           _p(tris), _p(roots, C.c_int32), _p(bounds)))
    return {"nodes": nodes, "triangles": tris, "roots": roots, "bounds": bounds}


def ref_body_poses_to_matrices(body_of_instance, local_pose, scale, bodies_per_world, worlds, poses):
    lib = ref_lib()
    b = np.ascontiguousarray(body_of_instance, np.int32)
    lp = np.ascontiguousarray(local_pose, np.float32)
    sc = np.ascontiguousarray(scale, np.float32)
    p = np.ascontiguousarray(poses, np.float32)
    out = np.zeros((worlds, len(b), 3, 4), np.float32)
    _ref_check(lib, lib.ngref_body_poses_to_matrices(int(bodies_per_world), _p(b, C.c_int32), _p(lp), _p(sc), len(b),
                                                     int(worlds), _p(p), _p(out)))
    return out


def ref_make_icosphere(radius, subdivisions):
    lib = ref_lib()
    nv, ni = C.c_int(), C.c_int()
    _ref_check(lib, lib.ngref_make_icosphere(float(radius), int(subdivisions), C.byref(nv), C.byref(ni), None, None))
    v = np.zeros((nv.value, 3), np.float32)
    i = np.zeros(ni.value, np.uint32)
    _ref_check(lib, lib.ngref_make_icosphere(float(radius), int(subdivisions), C.byref(nv), C.byref(ni), _p(v),
                                             _p(i, C.c_uint32)))
    return Mesh(v, i.reshape(-1, 3))


def ref_make_box(half):
    lib = ref_lib()
    v = np.zeros((8, 3), np.float32)
    i = np.zeros(36, np.uint32)
    lib.ngref_make_box(float(half[0]), float(half[1]), float(half[2]), _p(v), _p(i, C.c_uint32))
    return Mesh(v, i.reshape(-1, 3))


def ref_make_transform(position, rotation, scale):
    lib = ref_lib()
    p = np.asarray(position, np.float32)
    q = np.asarray(rotation, np.float32)
    out = np.zeros(12, np.float32)
    _ref_check(lib, lib.ngref_make_transform(_p(p), _p(q), float(scale), _p(out)))
    return out.reshape(3, 4)


def ref_camera_matrix(position, target, world_up=(0, 1, 0), fov=1.0, width=64, height=64):
    lib = ref_lib()
    out = np.zeros(12, np.float32)
    lib.ngref_camera_matrix(_p(np.asarray(position, np.float32)), _p(np.asarray(target, np.float32)),
                            _p(np.asarray(world_up, np.float32)), float(fov), int(width), int(height), _p(out))
    return out.reshape(3, 4)


def ref_make_camera(position, target, world_up=(0, 1, 0), fov=1.0, width=64, height=64):
    """The reference's make_camera: 14 floats (position, right, up, forward, fov_scale, aspect)."""
    lib = ref_lib()
    lib.ngref_make_camera.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_int, C.c_int, _f32p]
    out = np.zeros(14, np.float32)
    lib.ngref_make_camera(_p(np.asarray(position, np.float32)), _p(np.asarray(target, np.float32)),
                          _p(np.asarray(world_up, np.float32)), float(fov), int(width), int(height), _p(out))
    return out


def ref_invert_affine(m):
    lib = ref_lib()
    a = np.ascontiguousarray(m, np.float32).reshape(12)
    out = np.zeros(12, np.float32)
    ok = lib.ngref_invert_affine(_p(a), _p(out))
    return bool(ok), out.reshape(3, 4)


def ref_transform_aabb(m, box):
    lib = ref_lib()
    out = np.zeros(6, np.float32)
    lib.ngref_transform_aabb(_p(np.ascontiguousarray(m, np.float32).reshape(12)),
                             _p(np.ascontiguousarray(box, np.float32)), _p(out))
    return out
