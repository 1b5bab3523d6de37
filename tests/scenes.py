"""Scenes the tests share, after the reference's own batch tests (tests/test_batch.cpp, tests/test_batch.py).

Placements use numpy's seeded generator in the ranges the reference's tests use; the known-answer scenes
(one box per world, coincident boxes, a single instance) are placed exactly as the reference's tests place
them, so their known depths hold.
"""

from __future__ import annotations

import numpy as np

from neraulgraphics_b200.scene import (Instance, Light, Mesh, Plane, SceneDesc, Sphere, make_box, make_camera,
                                       make_icosphere, make_material, make_transform)

W, H = 96, 54
FOV = 1.5708
MAT = make_material((0.7, 0.5, 0.3), 0.9, 0.3, 0.0, 40.0)


def template(worlds=6, cameras_per_world=1):
    """A box, a ball and a smooth ball per world; a mirror sphere; two hard-shadow lights; a checker floor
    (tests/test_batch.cpp:75-119)."""
    smooth = make_icosphere(1.0, 2)
    smooth = Mesh(smooth.vertices, smooth.triangles, normals=smooth.vertices)
    meshes = [make_box((1, 1, 1)), make_icosphere(1.0, 2), smooth]
    instances = [Instance(0, material=MAT), Instance(1, material=make_material((0.2, 0.6, 0.3), 0.9, 0.3, 0, 40)),
                 Instance(2, material=make_material((0.3, 0.3, 0.8), 0.9, 0.3, 0, 40))]
    spheres = [Sphere((0, -1.0, -9), 1.0, make_material((0.8, 0.8, 0.9), 0.0, 10, 0.8, 800))]
    lights = [Light((-10, 10, 10), 1.4, 0.0), Light((15, 20, -5), 0.8, 0.0)]
    floor = Plane(y=-2, half_extent_x=30, z_min=-60, z_max=5, checker_scale=1,
                  material=make_material((1, 1, 1), 1, 0, 0, 1))
    return SceneDesc(W, H, worlds, cameras_per_world, spheres=spheres, lights=lights, floor=floor, meshes=meshes,
                     instances=instances)


def template_matrices(worlds, per_world=3, seed=3):
    rng = np.random.default_rng(seed)
    out = np.empty((worlds, per_world, 3, 4), np.float32)
    for w in range(worlds):
        for i in range(per_world):
            pos = (-3 + 2.5 * i + rng.random() - 0.5, rng.random() - 0.5 - 0.3 * (w % 7), -6 - 3 * rng.random())
            q = (rng.random() - 0.5, rng.random() - 0.5, rng.random() - 0.5, 1.0)
            out[w, i] = make_transform(pos, q, 0.6 + 0.6 * rng.random()).matrix
    return out


def camera(eye=(0, 0.5, 0), target=(0, 0, -8), width=W, height=H, fov=FOV):
    return make_camera(eye, target, width=width, height=height, fov=fov).matrix


def one_box_worlds():
    """Two worlds, one box each, at z = -8 and z = -3 (tests/test_batch.cpp:183-208)."""
    desc = SceneDesc(W, H, 2, 1, lights=[Light((0, 5, 5), 1.0, 0.0)], meshes=[make_box((1, 1, 1))],
                     instances=[Instance(0, material=MAT)])
    mats = np.stack([make_transform((0, 0, z)).matrix for z in (-8.0, -3.0)]).reshape(2, 1, 3, 4)
    cams = np.stack([camera((0, 0, 0), (0, 0, -1))] * 2)
    return desc, mats, cams


def single_leaf_worlds():
    """Four worlds of one box each at z = -4 - w: the tree is a single leaf (tests/test_batch.cpp:307-319)."""
    desc = SceneDesc(W, H, 4, 1, lights=[Light((-10, 10, 10), 1.4, 0.0)], meshes=[make_box((1, 1, 1))],
                     instances=[Instance(0, material=MAT)])
    mats = np.stack([make_transform((0, 0, -4.0 - w)).matrix for w in range(4)]).reshape(4, 1, 3, 4)
    cams = np.stack([camera((0, 0, 0), (0, 0, -8))] * 4)
    return desc, mats, cams


def coincident_boxes():
    """A thousand identical boxes in one world at z = -5: the nearest face is 4.8 away
    (tests/test_batch.cpp:321-331)."""
    desc = SceneDesc(W, H, 1, 1, lights=[Light((-10, 10, 10), 1.4, 0.0)], meshes=[make_box((0.2, 0.2, 0.2))],
                     instances=[Instance(0, material=MAT) for _ in range(1000)])
    mats = np.stack([make_transform((0.0, 0.0, -5.0)).matrix] * 1000).reshape(1, 1000, 3, 4)
    cams = camera((0, 0, 0), (0, 0, -8)).reshape(1, 3, 4)
    return desc, mats, cams


def scattered_boxes(worlds, per_world, seed=777):
    """Boxes and balls scattered through each world (tests/test_batch.cpp:335-374)."""
    meshes = [make_box((0.4, 0.4, 0.4)), make_icosphere(0.5, 1)]
    desc = SceneDesc(W, H, worlds, 1, lights=[Light((-10, 10, 10), 1.4, 0.0)], meshes=meshes,
                     instances=[Instance(i % 2, material=MAT) for i in range(per_world)])
    rng = np.random.default_rng(seed)
    spread = 60.0 if worlds == 1 else 3.0
    mats = np.empty((worlds, per_world, 3, 4), np.float32)
    for w in range(worlds):
        for i in range(per_world):
            pos = (spread * (rng.random() - 0.5), spread * 0.5 * (rng.random() - 0.5), -10.0 - spread * rng.random())
            q = (rng.random() - 0.5, rng.random() - 0.5, rng.random() - 0.5, 1.0)
            mats[w, i] = make_transform(pos, q, 0.5 + rng.random()).matrix
    cams = np.stack([camera((0, 0, 5), (0, 0, -30))] * worlds)
    return desc, mats, cams
