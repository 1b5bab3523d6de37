"""Seeded synthetic scenes for the batched sensor-rendering path.

The reference benchmarks on recorded simulator poses that are not available offline, so these seeded
scenes stand in for them, with the sizes and value distributions of the workloads the path is measured
on. Every generator is deterministic in its seed (numpy's default_rng).

- `icosphere_worlds`: 16 worlds at 64x64, each a floor and 8 icospheres (320 triangles) placed by matrices.
- `body_worlds`: 4096 worlds at 64x64, 20 simulator bodies each carrying one instance of three shared
  meshes (icosphere 1280, box 12, capped cylinder 512 triangles), moved by a Gaussian random walk.
- `uneven_worlds`: 2048 worlds of 1 to 200 instances of six meshes at 32x32, 64x64 or 128x128.
- `differentiable_worlds`: 1024 worlds at 128x128 of 12 icospheres and boxes, with target poses, for the adjoint.
- `large_world`: one world of 100,000 instances of five meshes at 1280x720, with a 64 x 2048 LiDAR sweep.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .scene import (Instance, Light, Material, Plane, SceneDesc, cylinder, make_box, make_camera, make_icosphere,
                    make_transform)

LIGHT = Light((-10.0, 20.0, 10.0), 1.6, 1.0)


@dataclass
class Workload:
    name: str
    desc: SceneDesc
    cameras: np.ndarray                      # (views, 3, 4) float32
    fov: float = 1.0
    spp: int = 1
    rgb: bool = True
    depth: bool = True
    normals: bool = False
    object_ids: bool = True
    matrices: np.ndarray | None = None       # (worlds, per_world, 3, 4) when placed by matrices
    binding: dict | None = None              # bind_bodies arguments when placed by bodies
    poses: np.ndarray | None = None          # (worlds, bodies, 7) initial body poses
    info: dict = field(default_factory=dict)


def uniform_quaternions(rng, n) -> np.ndarray:
    """n unit quaternions (x, y, z, w), uniform on S^3: normalised 4-d Gaussians."""
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def camera_matrix(position, target, width, height, fov) -> np.ndarray:
    return make_camera(position, target, width=width, height=height, fov=fov).matrix


def icosphere_worlds(worlds=16, per_world=8, width=64, height=64, seed=0) -> Workload:
    """16 worlds x 8 icospheres (subdivision 2, radius 0.5) over a floor, placed by matrices.

    Floor y = -2, half-extent 12 in x, z in (-30, -2), no checker. Per instance: position U[-2, 2]^3 + (0, 0, -6),
    rotation uniform on S^3, uniform scale U[0.5, 1.5]. One camera per world at (0, 1, 0) + U[-0.2, 0.2]^3 aimed at
    (0, 0, -6); fov 1.0 rad. One light at (-10, 20, 10), intensity 1.6, radius 1.0. Reflectivity 0.
    """
    rng = np.random.default_rng(seed)
    meshes = [make_icosphere(0.5, 2)]
    instances = [Instance(0, material=Material()) for _ in range(per_world)]
    floor = Plane(y=-2.0, half_extent_x=12.0, z_min=-30.0, z_max=-2.0, checker_scale=0.0)
    desc = SceneDesc(width, height, worlds, 1, lights=[LIGHT], floor=floor, meshes=meshes, instances=instances)
    mats = np.empty((worlds, per_world, 3, 4), np.float32)
    for w in range(worlds):
        pos = rng.uniform(-2.0, 2.0, size=(per_world, 3)) + np.array([0.0, 0.0, -6.0])
        q = uniform_quaternions(rng, per_world)
        sc = rng.uniform(0.5, 1.5, size=per_world)
        for i in range(per_world):
            mats[w, i] = make_transform(pos[i], q[i], sc[i]).matrix
    cams = np.empty((worlds, 3, 4), np.float32)
    for w in range(worlds):
        eye = np.array([0.0, 1.0, 0.0]) + rng.uniform(-0.2, 0.2, size=3)
        cams[w] = camera_matrix(eye, (0.0, 0.0, -6.0), width, height, 1.0)
    return Workload("icosphere_worlds", desc, cams, 1.0, 1, matrices=mats,
                    info={"worlds": worlds, "per_world": per_world, "width": width, "height": height, "seed": seed,
                          "triangles_per_instance": 320})


PALETTE = [(0.80, 0.25, 0.20), (0.20, 0.55, 0.80), (0.25, 0.70, 0.30), (0.85, 0.75, 0.20), (0.60, 0.30, 0.75),
           (0.90, 0.50, 0.15), (0.30, 0.75, 0.70), (0.75, 0.75, 0.75)]


def body_worlds(worlds=4096, bodies=20, width=64, height=64, seed=0) -> Workload:
    """4096 worlds x 20 bodies, one instance per body, of three shared meshes.

    Meshes: icosphere radius 0.5 subdivision 3 (1280 triangles), box of half-extent 0.4 (12), capped cylinder
    radius 1 half-height 1 with 128 segments (512). Instance i uses mesh i % 3 and sits on body i with a
    local offset U[-0.1, 0.1]^3 and a random local rotation; scale: icospheres U[0.6, 1.2] (uniform), boxes
    U[0.6, 1.2]^3, cylinders (0.3, 0.3, 0.5) * U[0.8, 1.2]. Initial body positions U[-2, 2]^3, rotations
    uniform on S^3. Floor y = -2.5, half-extent 8, z in (-8, 8), checker 1. Cameras: one per world on a
    ring of radius 4 at height 1.0, world w at angle 2 pi w / worlds, looking at the origin; fov 1.0 rad.
    Light as in icosphere_worlds. Outputs RGB, depth and object IDs, 1 sample per pixel.
    """
    rng = np.random.default_rng(seed)
    meshes = [make_icosphere(0.5, 3), make_box((0.4, 0.4, 0.4)), cylinder(1.0, 1.0, 128)]
    instances = [Instance(i % 3, material=Material(diffuse_color=PALETTE[i % len(PALETTE)])) for i in range(bodies)]
    floor = Plane(y=-2.5, half_extent_x=8.0, z_min=-8.0, z_max=8.0, checker_scale=1.0)
    desc = SceneDesc(width, height, worlds, 1, lights=[LIGHT], floor=floor, meshes=meshes, instances=instances)
    local = np.zeros((bodies, 7), np.float32)
    local[:, :3] = rng.uniform(-0.1, 0.1, size=(bodies, 3))
    local[:, 3:] = uniform_quaternions(rng, bodies)
    scale = np.zeros((bodies, 3), np.float32)
    for i in range(bodies):
        if i % 3 == 0:
            scale[i] = rng.uniform(0.6, 1.2)
        elif i % 3 == 1:
            scale[i] = rng.uniform(0.6, 1.2, size=3)
        else:
            scale[i] = np.array([0.3, 0.3, 0.5]) * rng.uniform(0.8, 1.2)
    binding = dict(body_of_instance=np.arange(bodies, dtype=np.int32), local_pose=local, scale=scale,
                   bodies_per_world=bodies)
    poses = np.zeros((worlds, bodies, 7), np.float32)
    poses[..., :3] = rng.uniform(-2.0, 2.0, size=(worlds, bodies, 3))
    poses[..., 3:] = uniform_quaternions(rng, worlds * bodies).reshape(worlds, bodies, 4)
    cams = np.empty((worlds, 3, 4), np.float32)
    for w in range(worlds):
        a = 2.0 * np.pi * w / worlds
        cams[w] = camera_matrix((4.0 * np.cos(a), 1.0, 4.0 * np.sin(a)), (0.0, 0.0, 0.0), width, height, 1.0)
    return Workload("body_worlds", desc, cams, 1.0, 1, binding=binding, poses=poses,
                    info={"worlds": worlds, "bodies": bodies, "width": width, "height": height, "seed": seed,
                          "triangles": [1280, 12, 512]})


def uneven_worlds(worlds=2048, seed=0):
    """2048 worlds of uneven sizes: instance counts uniform in 1..200, images of 32x32, 64x64 or 128x128.

    Six shared meshes: box of half-extent 0.4 (12 triangles), icosphere radius 0.5 subdivision 2 (320), capped
    cylinder radius 1 half-height 1 with 128 segments (512) at scale (0.3, 0.3, 0.5), icosphere subdivision 3
    (1280), 4 (5120) and 5 (20480). Instance i of a world uses mesh i % 6 with colour PALETTE[i % 8], so worlds
    of the same instance count hold the same instance list (they can share a plain renderer). Each instance is
    its own body: position uniform in [-r, r]^3 with r = 2 (count / 20)^(1/3) (the density of body_worlds),
    rotation uniform on S^3, uniform scale U[0.6, 1.2] (the cylinder's as above); the random walk of body_worlds
    moves them (walk_uneven). One camera per world on a ring of radius 2 r at height r / 2, world w at angle
    2 pi w / worlds, looking at the origin; fov 1.0 rad. Floor y = -r - 0.5, half-extent 4 r, z in (-4 r, 4 r),
    checker 1. Light as in icosphere_worlds (one floor and light for all worlds: the floor's placement follows
    the largest r).
    """
    rng = np.random.default_rng(seed)
    meshes = [make_box((0.4, 0.4, 0.4)), make_icosphere(0.5, 2), cylinder(1.0, 1.0, 128), make_icosphere(0.5, 3),
              make_icosphere(0.5, 4), make_icosphere(0.5, 5)]
    counts = rng.integers(1, 201, size=worlds)
    res = np.array([32, 64, 128])[rng.integers(0, 3, size=worlds)]
    spec, pos, quat, scale, cams = [], [], [], [], []
    rmax = 2.0 * (200 / 20.0) ** (1.0 / 3.0)
    for w in range(worlds):
        c, size = int(counts[w]), int(res[w])
        r = 2.0 * (c / 20.0) ** (1.0 / 3.0)
        insts = [Instance(i % 6, material=Material(diffuse_color=PALETTE[i % len(PALETTE)])) for i in range(c)]
        spec.append((size, size, insts))
        pos.append(rng.uniform(-r, r, size=(c, 3)))
        quat.append(uniform_quaternions(rng, c))
        sc = np.repeat(rng.uniform(0.6, 1.2, size=(c, 1)), 3, axis=1)
        sc[2::6] = np.array([0.3, 0.3, 0.5]) * sc[2::6]
        scale.append(sc)
        a = 2.0 * np.pi * w / worlds
        cams.append(camera_matrix((2 * r * np.cos(a), r / 2, 2 * r * np.sin(a)), (0.0, 0.0, 0.0), size, size, 1.0))
    floor = Plane(y=-rmax - 0.5, half_extent_x=4 * rmax, z_min=-4 * rmax, z_max=4 * rmax, checker_scale=1.0)
    pos, quat, scale = (np.concatenate(x).astype(np.float32) for x in (pos, quat, scale))
    return {"worlds": spec, "meshes": meshes, "floor": floor, "lights": [LIGHT], "cameras": np.stack(cams).astype(np.float32),
            "positions": pos, "quaternions": quat, "scales": scale, "counts": counts, "resolutions": res,
            "fov": 1.0, "seed": seed}


def walk_uneven(wl, steps, seed=1, sigma_pos=0.02, sigma_rot=0.05) -> np.ndarray:
    """(steps, total_instances, 3, 4) matrices of uneven_worlds' instances after each step of the random walk of
    body_worlds (random_walk), every instance its own body."""
    poses = np.concatenate([wl["positions"], wl["quaternions"]], -1)[None]
    walk = random_walk(poses, steps, seed=seed, sigma_pos=sigma_pos, sigma_rot=sigma_rot)[:, 0]
    return pose_matrices_np(walk[..., :3], walk[..., 3:], wl["scales"])


def differentiable_worlds(worlds=1024, per_world=12, width=128, height=128, seed=0) -> Workload:
    """1024 worlds at 128x128, depth and normals, for the adjoint: 12 instances each of an icosphere (radius 0.5,
    subdivision 3, 1280 triangles, smooth normals) and a box (half-extent 0.4, 12 triangles), alternating.

    Per instance: position U[-2, 2]^3 + (0, 0, -6), rotation uniform on S^3, uniform scale U[0.6, 1.2]. Floor
    y = -2.5, half-extent 12, z in (-30, -2). One camera per world at (0, 1, 0) + U[-0.2, 0.2]^3 aimed at
    (0, 0, -6), fov 1.0 rad. The target: the same scene with positions moved by N(0, 0.01^2) and each rotation
    turned by an angle N(0, 0.02^2) about a random axis. info holds positions (W, N, 3), quaternions (W, N, 4),
    scales (W, N, 3) and the target's positions and quaternions; matrices are the poses' (W, N, 3, 4).
    """
    rng = np.random.default_rng(seed)
    meshes = [make_icosphere(0.5, 3), make_box((0.4, 0.4, 0.4))]
    instances = [Instance(i % 2, material=Material(diffuse_color=PALETTE[i % len(PALETTE)])) for i in range(per_world)]
    floor = Plane(y=-2.5, half_extent_x=12.0, z_min=-30.0, z_max=-2.0, checker_scale=0.0)
    desc = SceneDesc(width, height, worlds, 1, lights=[LIGHT], floor=floor, meshes=meshes, instances=instances)
    pos = (rng.uniform(-2.0, 2.0, size=(worlds, per_world, 3)) + np.array([0.0, 0.0, -6.0])).astype(np.float32)
    quat = uniform_quaternions(rng, worlds * per_world).reshape(worlds, per_world, 4).astype(np.float32)
    scale = np.repeat(rng.uniform(0.6, 1.2, size=(worlds, per_world, 1)), 3, axis=-1).astype(np.float32)
    tpos = (pos + rng.normal(0.0, 0.01, size=pos.shape)).astype(np.float32)
    axis = rng.normal(size=pos.shape)
    axis /= np.linalg.norm(axis, axis=-1, keepdims=True)
    ang = rng.normal(0.0, 0.02, size=pos.shape[:-1] + (1,))
    tquat = quat_mul(quat.astype(np.float64), np.concatenate([axis * np.sin(ang / 2), np.cos(ang / 2)], -1))
    tquat = (tquat / np.linalg.norm(tquat, axis=-1, keepdims=True)).astype(np.float32)
    cams = np.empty((worlds, 3, 4), np.float32)
    for w in range(worlds):
        eye = np.array([0.0, 1.0, 0.0]) + rng.uniform(-0.2, 0.2, size=3)
        cams[w] = camera_matrix(eye, (0.0, 0.0, -6.0), width, height, 1.0)
    return Workload("differentiable_worlds", desc, cams, 1.0, 1, rgb=False, depth=True, normals=True, object_ids=False,
                    matrices=pose_matrices_np(pos, quat, scale),
                    info={"worlds": worlds, "per_world": per_world, "width": width, "height": height, "seed": seed,
                          "positions": pos, "quaternions": quat, "scales": scale, "target_positions": tpos,
                          "target_quaternions": tquat})


def pose_matrices_np(pos, quat, scale) -> np.ndarray:
    """[R(q) diag(s) | p] in float32, q normalised first (the arithmetic of autodiff.pose_matrices)."""
    q = quat.astype(np.float32)
    q = q / np.sqrt((q * q).sum(-1, keepdims=True))
    x, y, z, w = np.moveaxis(q, -1, 0)
    r = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                  2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                  2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)
    r = r.reshape(q.shape[:-1] + (3, 3)) * scale[..., None, :]
    return np.concatenate([r, pos[..., None]], -1).astype(np.float32)


def large_world(instances=100_000, width=1280, height=720, seed=0, frames=1) -> Workload:
    """One world of 100,000 instances of five meshes, rendered at 1280x720 and swept by a LiDAR.

    Meshes: box of half-extent 0.4 (12 triangles), icosphere radius 0.5 subdivision 2 (320), capped cylinder
    radius 1 half-height 1 with 128 segments (512) at scale (0.3, 0.3, 0.5), icosphere subdivision 3 (1280),
    icosphere subdivision 5 (20480); instance i uses mesh i % 5. Positions uniform in the box
    [-100, 100] x [-10, 10] x [-100, 100], rotations uniform on S^3, drawn afresh every frame (matrices:
    (frames, 1, instances, 3, 4)). Floor y = -11, half-extent 120, z in (-120, 120), checker 1. Camera at
    (0, 2, -100) looking at the origin, fov 1.0 rad. Light as in icosphere_worlds. info["lidar"]: 64
    elevations in [-15, 15] degrees x 2048 azimuths from the scene centre, max range 150.
    """
    rng = np.random.default_rng(seed)
    meshes = [make_box((0.4, 0.4, 0.4)), make_icosphere(0.5, 2), cylinder(1.0, 1.0, 128), make_icosphere(0.5, 3),
              make_icosphere(0.5, 5)]
    insts = [Instance(i % 5, material=Material(diffuse_color=PALETTE[i % len(PALETTE)])) for i in range(instances)]
    floor = Plane(y=-11.0, half_extent_x=120.0, z_min=-120.0, z_max=120.0, checker_scale=1.0)
    desc = SceneDesc(width, height, 1, 1, lights=[LIGHT], floor=floor, meshes=meshes, instances=insts)
    mats = np.empty((frames, 1, instances, 3, 4), np.float32)
    scale = np.ones((instances, 3))
    scale[2::5] = (0.3, 0.3, 0.5)
    for f in range(frames):
        pos = rng.uniform((-100.0, -10.0, -100.0), (100.0, 10.0, 100.0), size=(instances, 3))
        q = uniform_quaternions(rng, instances)
        x, y, z, w = q.T
        r = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                      2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                      2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1).reshape(instances, 3, 3)
        mats[f, 0, :, :, :3] = r * scale[:, None, :]
        mats[f, 0, :, :, 3] = pos
    cams = camera_matrix((0.0, 2.0, -100.0), (0.0, 0.0, 0.0), width, height, 1.0)[None]
    el = np.radians(np.linspace(-15.0, 15.0, 64))
    az = np.radians(np.linspace(0.0, 360.0, 2048, endpoint=False))
    e, a = np.meshgrid(el, az, indexing="ij")
    dirs = np.stack([np.cos(e) * np.sin(a), np.sin(e), np.cos(e) * np.cos(a)], -1).reshape(1, -1, 3).astype(np.float32)
    origins = np.zeros_like(dirs)
    return Workload("large_world", desc, cams.astype(np.float32), 1.0, 1, matrices=mats,
                    info={"instances": instances, "width": width, "height": height, "seed": seed,
                          "triangles": [12, 320, 512, 1280, 20480], "lidar": {"origins": origins, "directions": dirs,
                                                                             "max_distance": 150.0}})


def quat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Hamilton product of (..., 4) quaternions stored (x, y, z, w)."""
    ax, ay, az, aw = np.moveaxis(a, -1, 0)
    bx, by, bz, bw = np.moveaxis(b, -1, 0)
    return np.stack([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], axis=-1)


def random_walk(poses: np.ndarray, steps: int, seed=1, sigma_pos=0.02, sigma_rot=0.05) -> np.ndarray:
    """(steps, worlds, bodies, 7): each step adds N(0, sigma_pos^2) to every position and turns every body by an
    angle N(0, sigma_rot^2) about a random unit axis (q <- q * dq)."""
    rng = np.random.default_rng(seed)
    cur = poses.astype(np.float64).copy()
    out = np.empty((steps,) + poses.shape, np.float32)
    for s in range(steps):
        cur[..., :3] += rng.normal(0.0, sigma_pos, size=cur[..., :3].shape)
        axis = rng.normal(size=cur[..., :3].shape)
        axis /= np.linalg.norm(axis, axis=-1, keepdims=True)
        ang = rng.normal(0.0, sigma_rot, size=cur.shape[:-1] + (1,))
        dq = np.concatenate([axis * np.sin(ang / 2), np.cos(ang / 2)], axis=-1)
        q = quat_mul(cur[..., 3:], dq)
        cur[..., 3:] = q / np.linalg.norm(q, axis=-1, keepdims=True)
        out[s] = cur
    return out
