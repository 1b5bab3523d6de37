"""neraulgraphics_b200: a B200-native (sm_100a) batched multi-world sensor renderer.

A drop-in for neraulgraphics' BatchRenderer path: many worlds of the same instances, each seen by its own
cameras, rendered into RGB, depth, normal and object-ID images in one launch on one GPU. The names below
mirror the reference's Python module (python/bindings.cpp, python/neraulgraphics/shapes.py).
"""

from __future__ import annotations

import ctypes as _C

import numpy as _np

from . import _abi
from ._abi import (MAX_LIGHTS, MAX_SPHERES, OBJECT_FLOOR, OBJECT_INSTANCE, OBJECT_NONE, OBJECT_SPHERE,
                   OUTPUT_DEPTH, OUTPUT_NORMAL, OUTPUT_OBJECT_ID, OUTPUT_RGB)
from ._lib import CudaError, DeviceTimeout
from .renderer import BatchRenderer, Renderer, UnevenBatchRenderer
from .scene import (Camera, Environment, Instance, Light, Material, Mesh, Plane, SceneDesc, Sphere, Transform, cylinder,
                    identity_transform, look_at, make_box, make_camera, make_icosphere, make_material, make_transform)

__version__ = "0.1.0"


def device_bytes() -> int:
    """Bytes of device memory held by every renderer of the process (ngb_device_bytes)."""
    from ._lib import lib
    return int(lib().ngb_device_bytes())


def inject_allocation_failure(after: int = 0) -> None:
    """Testing: the after-th device allocation from now on fails as an out-of-memory cudaMalloc would (the call
    raises CudaError and the renderer stays usable); after < 0 cancels (ngb_inject_allocation_failure)."""
    from ._lib import lib
    lib().ngb_inject_allocation_failure(int(after))


def cuda_available() -> bool:
    """True when a CUDA GPU is present (there is no CPU backend)."""
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def build_meshes(meshes) -> dict:
    """The meshes' bottom-level trees as the renderer builds them (host only): nodes (N, 8) int32 words,
    triangles (T, 12) float32, roots, bounds (M, 6), triangle_index (T,)."""
    from ._lib import check, lib
    L = lib()
    desc = SceneDesc(1, 1, 1, meshes=meshes)
    nn, nt = _C.c_int32(), _C.c_int32()
    check(L.ngb_build_meshes(desc.c.meshes, len(meshes), _C.byref(nn), _C.byref(nt), None, None, None, None, None))
    nodes = _np.zeros((nn.value, 8), _np.int32)
    tris = _np.zeros((nt.value, 12), _np.float32)
    roots = _np.zeros(len(meshes), _np.int32)
    bounds = _np.zeros((len(meshes), 6), _np.float32)
    tidx = _np.zeros(nt.value, _np.int32)
    vp = lambda a: a.ctypes.data_as(_C.c_void_p)
    check(L.ngb_build_meshes(desc.c.meshes, len(meshes), _C.byref(nn), _C.byref(nt), vp(nodes), vp(tris), vp(roots),
                             vp(bounds), vp(tidx)))
    return {"nodes": nodes, "triangles": tris, "roots": roots, "bounds": bounds, "triangle_index": tidx}
