"""Loads libngb.so and declares its C ABI (include/ngb.h) for ctypes.

There is no fallback: if the library is missing or cannot load, every use raises.
"""

from __future__ import annotations

import ctypes as C
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libngb.so")

_lib = None

_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_vp = C.c_void_p


class CudaError(RuntimeError):
    """A failed CUDA call or device fault (neraulgraphics.CudaError in the reference)."""


class DeviceTimeout(CudaError):
    """A bounded wait on the GPU ran out."""


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CudaError(f"{LIB_PATH} is not built; run `python -m neraulgraphics_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.ngb_create.argtypes = [C.POINTER(_abi.SceneC), C.POINTER(_vp)]
    L.ngb_create_uneven.argtypes = [C.POINTER(_abi.SceneC), C.POINTER(_abi.UnevenWorldC), C.c_int32, C.POINTER(_vp)]
    L.ngb_pixel_count.restype = C.c_int64
    L.ngb_pixel_count.argtypes = [_vp]
    L.ngb_destroy.argtypes = [_vp]
    L.ngb_last_error.restype = C.c_char_p
    L.ngb_last_error.argtypes = [_vp]
    L.ngb_set_instance_transforms.argtypes = [_vp, _vp, C.c_int32]
    L.ngb_bind_bodies.argtypes = [_vp, C.c_int32, _i32p, _f32p, _f32p]
    L.ngb_set_body_poses.argtypes = [_vp, _vp, C.c_int32]
    L.ngb_bind_geoms.argtypes = [_vp, C.c_int32, _i32p, _f32p]
    L.ngb_set_geom_poses.argtypes = [_vp, _vp, _vp, C.c_int32]
    L.ngb_update_mesh.argtypes = [_vp, C.c_int32, _vp, _vp, C.c_int32]
    L.ngb_record_hits_into.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.ngb_pose_matrices.argtypes = [_vp, _vp, _vp, C.c_int64, _vp, _vp]
    L.ngb_pose_matrices_grad.argtypes = [_vp, _vp, C.c_int64, _vp, _vp, _vp, _vp, _vp]
    L.ngb_inspect_mesh.argtypes = [_vp, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp]
    L.ngb_render.argtypes = [_vp, _vp, C.c_float, C.c_int32, C.c_uint32, C.c_int32, C.c_int32,
                             C.POINTER(_abi.BatchFrameC)]
    L.ngb_render_into.argtypes = [_vp, _vp, C.c_float, C.c_int32, C.c_uint32, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp]
    L.ngb_render_host.argtypes = [_vp, _vp, C.c_float, C.c_int32, C.c_uint32, C.c_int32, _vp, _vp, _vp, _vp]
    L.ngb_cast_rays.argtypes = [_vp, _vp, _vp, C.c_int32, C.c_float, C.c_int32, C.POINTER(_abi.RayHitsC)]
    L.ngb_cast_rays_into.argtypes = [_vp, _vp, _vp, C.c_int32, C.c_float, C.c_int32, _vp, _vp, _vp]
    L.ngb_copy_to_host.argtypes = [_vp, _vp, _vp, C.c_size_t]
    L.ngb_set_ambient.argtypes = [_vp, C.c_float]
    L.ngb_ambient.restype = C.c_float
    L.ngb_ambient.argtypes = [_vp]
    L.ngb_set_environment.argtypes = [_vp, C.POINTER(_abi.EnvironmentC)]
    L.ngb_set_stream.argtypes = [_vp, _vp]
    L.ngb_set_sync.argtypes = [_vp, C.c_int32, C.c_double]
    L.ngb_synchronize.argtypes = [_vp, C.c_double]
    L.ngb_last_stage_ms.argtypes = [_vp, _f32p, C.c_int32, _i32p]
    for name in ("ngb_width", "ngb_height", "ngb_world_count", "ngb_cameras_per_world", "ngb_view_count",
                 "ngb_instances_per_world"):
        getattr(L, name).argtypes = [_vp]
        getattr(L, name).restype = C.c_int32
    L.ngb_last_kernel_ms.restype = C.c_float
    L.ngb_last_kernel_ms.argtypes = [_vp]
    L.ngb_build_meshes.argtypes = [C.POINTER(_abi.MeshC), C.c_int32, _i32p, _i32p, _vp, _vp, _vp, _vp, _vp]
    L.ngb_build_tlas_noalloc.argtypes = [C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.ngb_set_tuning.argtypes = [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.ngb_set_build.argtypes = [_vp, C.c_int32]
    L.ngb_set_tile_shape.argtypes = [_vp, C.c_int32, C.c_int32]
    L.ngb_set_ray_kernel.argtypes = [_vp, C.c_int32]
    L.ngb_make_camera.argtypes = [_abi.Vec3, _abi.Vec3, _abi.Vec3, C.c_float, C.c_int32, C.c_int32,
                                  C.POINTER(_abi.CameraC)]
    L.ngb_render_view.argtypes = [_vp, C.POINTER(_abi.CameraC), C.c_int32, C.c_int32, _vp]
    L.ngb_render_view_frame.argtypes = [_vp, C.POINTER(_abi.CameraC), C.c_int32, C.c_int32, C.c_uint32,
                                        C.POINTER(_abi.BatchFrameC)]
    L.ngb_view_pixels.argtypes = [_vp, C.POINTER(C.c_void_p)]
    L.ngb_set_lights.argtypes = [_vp, C.POINTER(_abi.LightC), C.c_int32]
    L.ngb_set_rows.argtypes = [_vp, C.c_int32, C.c_int32]
    L.ngb_device_bytes.argtypes = []
    L.ngb_device_bytes.restype = C.c_int64
    L.ngb_inject_allocation_failure.argtypes = [C.c_int32]
    L.ngb_rows.argtypes = [_vp, _i32p, _i32p]
    L.ngb_copy_hits.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.ngb_depth_normal_adjoint.argtypes = [_vp, _vp, _vp, C.c_float] + [_vp] * 9
    L.ngb_srgb_thresholds.argtypes = [_vp]
    L.ngb_record_hits.argtypes = [_vp, C.c_int32]
    L.ngb_inspect_tlas.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.ngb_inspect_hits.argtypes = [_vp, _vp, _vp, _vp, _vp]
    _lib = L
    return L


def check(status: int, handle=None) -> None:
    """Raises the Python exception for a status of the C ABI."""
    if status == _abi.NGB_OK:
        return
    msg = lib().ngb_last_error(handle).decode()
    if status == _abi.NGB_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == _abi.NGB_TIMEOUT:
        raise DeviceTimeout(msg)
    if status == _abi.NGB_LOGIC_ERROR:
        raise RuntimeError(msg)
    raise CudaError(msg)
