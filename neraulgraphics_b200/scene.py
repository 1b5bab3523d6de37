"""Scene description types, with the reference's Python names, fields and defaults.

They mirror the classes the reference's Python module exposes (python/bindings.cpp:384-640): Material,
Sphere, Light, Plane, Transform, Mesh, Instance, Environment, and the helpers make_transform,
identity_transform, make_box, make_icosphere and make_camera. They are plain Python data; `to_abi` packs a
scene into the structs of include/ngb.h.

The generators are written to give the same float32 bits as the reference's C++ (src/mesh.cpp,
src/renderer.cpp:39-59): every operation is done in the same precision and order.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

Vec3T = tuple


def _v3(v) -> tuple:
    t = tuple(float(x) for x in v)
    if len(t) != 3:
        raise ValueError(f"expected 3 numbers, got {len(t)}")
    return t


@dataclass
class Material:
    """How a surface reflects light (include/neraulgraphics/scene.h:35-56; python/bindings.cpp:384-406)."""
    diffuse_color: Vec3T = (0.8, 0.8, 0.8)
    diffuse_albedo: float = 0.9
    specular_albedo: float = 0.1
    reflectivity: float = 0.0
    specular_exponent: float = 50.0
    roughness: float = -1.0
    metallic: float = -1.0
    emission: Vec3T = (0.0, 0.0, 0.0)
    transmission: float = 0.0
    ior: float = 1.5

    def to_abi(self) -> _abi.MaterialC:
        return _abi.MaterialC(_abi.Vec3(*_v3(self.diffuse_color)), self.diffuse_albedo, self.specular_albedo,
                              self.reflectivity, self.specular_exponent, self.roughness, self.metallic,
                              _abi.Vec3(*_v3(self.emission)), self.transmission, self.ior)


def make_material(color, kd, ks, kr, exponent) -> Material:
    """include/neraulgraphics/scene.h:58-61."""
    return Material(tuple(color), kd, ks, kr, exponent)


@dataclass
class Sphere:
    center: Vec3T
    radius: float
    material: Material = field(default_factory=Material)


@dataclass
class Light:
    """A point or sphere light (scene.h:82-92). radius 0 gives hard shadows."""
    position: Vec3T
    intensity: float = 1.0
    radius: float = 0.0
    falloff: float = 0.0
    direction: Vec3T = (0.0, 0.0, -1.0)
    spot_angle: float = 0.0
    spot_softness: float = 0.25
    color: Vec3T = (1.0, 1.0, 1.0)


@dataclass
class Plane:
    """A finite checkerboard floor at constant y (scene.h:96-103). Plane() is no floor at all."""
    y: float = 0.0
    half_extent_x: float = 0.0
    z_min: float = 0.0
    z_max: float = 0.0
    checker_scale: float = 0.5
    material: Material = field(default_factory=lambda: Material((1.0, 1.0, 1.0), 1.0, 0.0, 0.0, 1.0))


@dataclass
class Environment:
    """The gradient sky (scene.h:109-121). Environment maps are not supported by this renderer."""
    up: Vec3T = (0.0, 1.0, 0.0)
    color_up: Vec3T = (0.10, 0.26, 0.60)
    color_down: Vec3T = (0.35, 0.52, 0.70)
    intensity: float = 1.0

    def to_abi(self) -> _abi.EnvironmentC:
        return _abi.EnvironmentC(_abi.Vec3(*_v3(self.up)), _abi.Vec3(*_v3(self.color_up)),
                                 _abi.Vec3(*_v3(self.color_down)), self.intensity)


class Transform:
    """An affine map as the top three rows of a 4x4 matrix, row-major (mesh.h:193-198)."""

    def __init__(self, matrix):
        m = np.asarray(matrix, dtype=np.float32)
        if m.ndim != 2 or m.shape[1] != 4 or m.shape[0] not in (3, 4):
            raise ValueError(f"transform matrix must be 3x4 or 4x4, got {'x'.join(map(str, m.shape))}")
        self._m = np.ascontiguousarray(m[:3]).copy()

    @property
    def matrix(self) -> np.ndarray:
        return self._m.copy()

    def __repr__(self):
        return f"Transform(position=({self._m[0, 3]}, {self._m[1, 3]}, {self._m[2, 3]}), ...)"


def identity_transform() -> Transform:
    return Transform(np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]], np.float32))


def make_transform(position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0), scale=1.0) -> Transform:
    """Scale, then rotate, then translate: the float arithmetic of make_transform (src/mesh.cpp:473-487)."""
    f = np.float32
    qx, qy, qz, qw = (f(v) for v in rotation)
    norm = np.sqrt(qx * qx + qy * qy + qz * qz + qw * qw)
    if not (norm > 0) or not np.isfinite(norm):
        raise ValueError("rotation quaternion must be finite and not zero")
    x, y, z, w = qx / norm, qy / norm, qz / norm, qw / norm
    s, one, two = f(scale), f(1), f(2)
    p = [f(v) for v in position]
    m = [s * (one - two * (y * y + z * z)), s * (two * (x * y - z * w)), s * (two * (x * z + y * w)), p[0],
         s * (two * (x * y + z * w)), s * (one - two * (x * x + z * z)), s * (two * (y * z - x * w)), p[1],
         s * (two * (x * z - y * w)), s * (two * (y * z + x * w)), s * (one - two * (x * x + y * y)), p[2]]
    return Transform(np.array(m, np.float32).reshape(3, 4))


class Mesh:
    """Triangles: (V, 3) float32 vertices, (T, 3) uint32 indices, optional (V, 3) vertex normals (mesh.h:160-171)."""

    def __init__(self, vertices, triangles, normals=None, uvs=None):
        if uvs is not None:
            raise ValueError("meshes with uvs (textures) are not supported by this renderer")
        self.vertices = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
        self.triangles = np.ascontiguousarray(np.asarray(triangles, np.uint32).reshape(-1, 3))
        self.normals = None if normals is None else np.ascontiguousarray(np.asarray(normals, np.float32).reshape(-1, 3))

    @property
    def triangle_count(self) -> int:
        return len(self.triangles)

    def __repr__(self):
        return f"Mesh({len(self.vertices)} vertices, {len(self.triangles)} triangles)"


@dataclass
class Instance:
    """A mesh placed in a world with its own transform and material (mesh.h:207-222)."""
    mesh: int
    transform: Transform = field(default_factory=identity_transform)
    material: Material = field(default_factory=Material)


def make_box(half_extents) -> Mesh:
    """An axis-aligned box centred on the origin, 12 triangles (src/mesh.cpp:489-503)."""
    hx, hy, hz = (np.float32(v) for v in half_extents)
    verts = [((hx if i & 1 else -hx), (hy if i & 2 else -hy), (hz if i & 4 else -hz)) for i in range(8)]
    idx = [0, 2, 1, 1, 2, 3, 4, 5, 6, 5, 7, 6, 0, 1, 4, 1, 5, 4, 2, 6, 3, 3, 6, 7, 0, 4, 2, 2, 4, 6, 1, 3, 5, 3, 7, 5]
    return Mesh(np.array(verts, np.float32), np.array(idx, np.uint32))


def make_icosphere(radius: float, subdivisions: int = 3) -> Mesh:
    """A subdivided icosahedron, 20 * 4**subdivisions triangles (src/mesh.cpp:505-553), in float32."""
    f = np.float32
    radius = f(radius)
    if not (radius > 0) or not np.isfinite(radius):
        raise ValueError(f"icosphere radius must be positive, got {float(radius):f}")
    if subdivisions < 0 or subdivisions > 8:
        raise ValueError(f"icosphere subdivisions must be 0 to 8, got {subdivisions}")
    verts: list = []

    def add(x, y, z):
        x, y, z = f(x), f(y), f(z)
        ln = np.sqrt(x * x + y * y + z * z)
        verts.append((x / ln, y / ln, z / ln))
        return len(verts) - 1

    t = (f(1) + np.sqrt(f(5))) / f(2)
    for p in [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
              (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]:
        add(*p)
    indices = [0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
               3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1]
    for _ in range(subdivisions):
        mids: dict = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key in mids:
                return mids[key]
            va, vb = verts[a], verts[b]
            mids[key] = add(va[0] + vb[0], va[1] + vb[1], va[2] + vb[2])
            return mids[key]

        nxt = []
        for i in range(0, len(indices), 3):
            a, b, c = indices[i], indices[i + 1], indices[i + 2]
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nxt += [a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca]
        indices = nxt
    v = np.array(verts, np.float32) * radius
    return Mesh(v, np.array(indices, np.uint32))


@dataclass
class Camera:
    position: tuple
    right: tuple
    up: tuple
    forward: tuple
    fov_scale: float
    aspect: float

    @property
    def matrix(self) -> np.ndarray:
        """The camera-to-world matrix (OpenGL convention) the batch API takes (tests/test_batch.cpp:59-62)."""
        r, u, fw, p = self.right, self.up, self.forward, self.position
        return np.array([[r[0], u[0], -fw[0], p[0]], [r[1], u[1], -fw[1], p[1]], [r[2], u[2], -fw[2], p[2]]],
                        np.float32)


def lights_abi(lights):
    """The lights as an ngb_light array (at least one entry long)."""
    lig = (_abi.LightC * max(1, len(lights)))()
    for i, l in enumerate(lights):
        lig[i] = _abi.LightC(_abi.Vec3(*_v3(l.position)), l.intensity, l.radius, l.falloff,
                             _abi.Vec3(*_v3(l.direction)), l.spot_angle, l.spot_softness, _abi.Vec3(*_v3(l.color)))
    return lig


_libm = None


def _tanf(x: float) -> float:
    """The C library's single-precision tangent, which std::tan(float) calls (numpy's float32 tan is its own)."""
    global _libm
    if _libm is None:
        import ctypes
        import ctypes.util
        _libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
        _libm.tanf.restype = ctypes.c_float
        _libm.tanf.argtypes = [ctypes.c_float]
    return float(_libm.tanf(x))


def make_camera(position, target, *, width: int, height: int, world_up=(0.0, 1.0, 0.0), fov=1.5707964) -> Camera:
    """A camera at position looking at target: the basis in double, then rounded (src/renderer.cpp:39-59)."""
    pos = [float(np.float32(v)) for v in position]
    tgt = [float(np.float32(v)) for v in target]
    wup = [float(np.float32(v)) for v in world_up]

    def norm(a):
        n = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
        return [a[0] / n, a[1] / n, a[2] / n]

    def cross(a, b):
        return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]

    fwd = norm([tgt[0] - pos[0], tgt[1] - pos[1], tgt[2] - pos[2]])
    right = norm(cross(fwd, wup))
    up = cross(right, fwd)
    f32 = lambda a: tuple(float(np.float32(x)) for x in a)
    fov_scale = _tanf(float(np.float32(np.float32(fov) * np.float32(0.5))))
    return Camera(f32(pos), f32(right), f32(up), f32(fwd), fov_scale, float(np.float32(width) / np.float32(height)))


def _revolve(profile: np.ndarray, segments: int) -> Mesh:
    """A (radius, z) profile spun round the Z axis (python/neraulgraphics/shapes.py:20-57)."""
    if segments < 3:
        raise ValueError(f"segments must be at least 3, got {segments}")
    angle = np.linspace(0.0, 2.0 * np.pi, segments, endpoint=False)
    cos, sin = np.cos(angle), np.sin(angle)
    rows, start, n = [], [], 0
    for radius, z in profile:
        start.append(n)
        if radius == 0.0:
            rows.append(np.array([[0.0, 0.0, z]]))
        else:
            rows.append(np.stack([radius * cos, radius * sin, np.full(segments, z)], axis=1))
        n += len(rows[-1])
    tris = []
    for row in range(len(profile) - 1):
        a_point, b_point = profile[row][0] == 0.0, profile[row + 1][0] == 0.0
        a, b = start[row], start[row + 1]
        for i in range(segments):
            j = (i + 1) % segments
            if a_point and b_point:
                continue
            if a_point:
                tris.append((a, b + i, b + j))
            elif b_point:
                tris.append((a + i, a + j, b))
            else:
                tris.append((a + i, a + j, b + j))
                tris.append((a + i, b + j, b + i))
    return Mesh(np.concatenate(rows).astype(np.float32), np.array(tris, dtype=np.uint32))


def cylinder(radius: float = 1.0, half_height: float = 1.0, segments: int = 32) -> Mesh:
    """A capped cylinder along Z (python/neraulgraphics/shapes.py:83-86): 4 * segments triangles."""
    return _revolve(np.array([[0, half_height], [radius, half_height], [radius, -half_height], [0, -half_height]],
                             dtype=np.float64), segments)


def look_at(eye, target, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """(N, 3, 4) camera-to-world matrices looking from eye to target (python/neraulgraphics/shapes.py:126-143)."""
    eye, target = np.broadcast_arrays(np.atleast_2d(np.asarray(eye, np.float64)),
                                      np.atleast_2d(np.asarray(target, np.float64)))
    forward = target - eye
    forward = forward / np.linalg.norm(forward, axis=1, keepdims=True)
    right = np.cross(forward, np.asarray(up, np.float64))
    nrm = np.linalg.norm(right, axis=1, keepdims=True)
    if (nrm < 1e-9).any():
        raise ValueError("a camera looks along the up axis, so its right direction is undefined; move the eye or change up")
    right = right / nrm
    true_up = np.cross(right, forward)
    out = np.empty((len(eye), 3, 4), dtype=np.float32)
    out[:, :, 0], out[:, :, 1], out[:, :, 2], out[:, :, 3] = right, true_up, -forward, eye
    return out


class SceneDesc:
    """A scene packed into the structs of include/ngb.h. Keeps the numpy arrays the pointers refer to alive."""

    def __init__(self, width, height, world_count, cameras_per_world=1, spheres=(), lights=(), floor=None,
                 meshes=(), instances=(), device=0):
        floor = floor if floor is not None else Plane()
        self.meshes = list(meshes)
        self.instances = list(instances)
        self._keep = []
        sph = (_abi.SphereC * max(1, len(spheres)))()
        for i, s in enumerate(spheres):
            sph[i] = _abi.SphereC(_abi.Vec3(*_v3(s.center)), s.radius, s.material.to_abi())
        lig = lights_abi(lights)
        msh = (_abi.MeshC * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            v = np.ascontiguousarray(m.vertices, np.float32)
            t = np.ascontiguousarray(m.triangles, np.uint32)
            nrm = None if m.normals is None else np.ascontiguousarray(m.normals, np.float32)
            self._keep += [v, t, nrm]
            msh[i] = _abi.MeshC(v.ctypes.data_as(C.POINTER(C.c_float)), len(v),
                                t.ctypes.data_as(C.POINTER(C.c_uint32)), t.size,
                                None if nrm is None else nrm.ctypes.data_as(C.POINTER(C.c_float)))
        ins = (_abi.InstanceC * max(1, len(self.instances)))()
        for i, inst in enumerate(self.instances):
            tr = inst.transform.matrix.reshape(-1) if isinstance(inst.transform, Transform) else \
                np.asarray(inst.transform, np.float32).reshape(-1)[:12]
            ins[i] = _abi.InstanceC(int(inst.mesh), (C.c_float * 12)(*[float(x) for x in tr]), inst.material.to_abi())
        self._keep += [sph, lig, msh, ins]
        fl = _abi.PlaneC(floor.y, floor.half_extent_x, floor.z_min, floor.z_max, floor.checker_scale,
                         floor.material.to_abi())
        self.c = _abi.SceneC(int(width), int(height), int(world_count), int(cameras_per_world),
                             sph, len(spheres), lig, len(lights), fl, msh, len(self.meshes), ins, len(self.instances),
                             int(device))
        self.width, self.height = int(width), int(height)
        self.world_count, self.cameras_per_world = int(world_count), int(cameras_per_world)
        self.spheres, self.lights, self.floor = list(spheres), list(lights), floor

    @property
    def view_count(self) -> int:
        return self.world_count * self.cameras_per_world

    @property
    def per_world(self) -> int:
        return len(self.instances)
