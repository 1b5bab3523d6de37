"""ctypes mirrors of the plain-C structs of include/ngb.h.

These are the only types that cross the C ABI. The product (libngb.so) takes them, and so do the
test-only checkers (the oracle and the reference harness), so one scene description drives all three.
"""

from __future__ import annotations

import ctypes as C

NGB_OK = 0
NGB_INVALID_ARGUMENT = 1
NGB_CUDA_ERROR = 2
NGB_TIMEOUT = 3
NGB_LOGIC_ERROR = 4

MEMORY_HOST = 0
MEMORY_DEVICE = 1

OUTPUT_RGB = 1
OUTPUT_DEPTH = 2
OUTPUT_NORMAL = 4
OUTPUT_OBJECT_ID = 8

MAX_SPHERES = 32
MAX_LIGHTS = 8
OBJECT_NONE = 0
OBJECT_SPHERE = 1
OBJECT_FLOOR = OBJECT_SPHERE + MAX_SPHERES
OBJECT_INSTANCE = OBJECT_FLOOR + 1


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class MaterialC(C.Structure):
    _fields_ = [("diffuse_color", Vec3), ("diffuse_albedo", C.c_float), ("specular_albedo", C.c_float),
                ("reflectivity", C.c_float), ("specular_exponent", C.c_float), ("roughness", C.c_float),
                ("metallic", C.c_float), ("emission", Vec3), ("transmission", C.c_float), ("ior", C.c_float)]


class SphereC(C.Structure):
    _fields_ = [("center", Vec3), ("radius", C.c_float), ("material", MaterialC)]


class LightC(C.Structure):
    _fields_ = [("position", Vec3), ("intensity", C.c_float), ("radius", C.c_float), ("falloff", C.c_float),
                ("direction", Vec3), ("spot_angle", C.c_float), ("spot_softness", C.c_float), ("color", Vec3)]


class PlaneC(C.Structure):
    _fields_ = [("y", C.c_float), ("half_extent_x", C.c_float), ("z_min", C.c_float), ("z_max", C.c_float),
                ("checker_scale", C.c_float), ("material", MaterialC)]


class MeshC(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("vertex_count", C.c_int32),
                ("indices", C.POINTER(C.c_uint32)), ("index_count", C.c_int32), ("normals", C.POINTER(C.c_float))]


class InstanceC(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("transform", C.c_float * 12), ("material", MaterialC)]


class EnvironmentC(C.Structure):
    _fields_ = [("up", Vec3), ("color_up", Vec3), ("color_down", Vec3), ("intensity", C.c_float)]


class SceneC(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("world_count", C.c_int32),
                ("cameras_per_world", C.c_int32), ("spheres", C.POINTER(SphereC)), ("sphere_count", C.c_int32),
                ("lights", C.POINTER(LightC)), ("light_count", C.c_int32), ("floor", PlaneC),
                ("meshes", C.POINTER(MeshC)), ("mesh_count", C.c_int32), ("instances", C.POINTER(InstanceC)),
                ("instance_count", C.c_int32), ("device", C.c_int32)]


class CameraC(C.Structure):
    """ngb_camera: neraulgraphics::Camera (include/neraulgraphics/scene.h:125-132)."""
    _fields_ = [("position", Vec3), ("right", Vec3), ("up", Vec3), ("forward", Vec3), ("fov_scale", C.c_float),
                ("aspect", C.c_float)]


class BatchFrameC(C.Structure):
    _fields_ = [("memory", C.c_int32), ("device_id", C.c_int32), ("views", C.c_int32), ("width", C.c_int32),
                ("height", C.c_int32), ("rgb", C.c_void_p), ("depth", C.c_void_p), ("normal", C.c_void_p),
                ("object_id", C.c_void_p)]


class RayHitsC(C.Structure):
    _fields_ = [("memory", C.c_int32), ("device_id", C.c_int32), ("count", C.c_int32), ("distance", C.c_void_p),
                ("normal", C.c_void_p), ("object_id", C.c_void_p)]


class UnevenWorldC(C.Structure):
    """ngb_uneven_world: one world of an uneven batch."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("instance_count", C.c_int32)]
