"""Generates the golden fixtures in this folder from the REFERENCE implementation itself.

    python tests/golden/make_golden.py

Needs oracle/_ref/libngref.so: neraulgraphics 0.5.0's own CPU backend, compiled from its sources by
`make -C oracle ref`. Each fixture holds a seeded scene's inputs and the images (and ray hits) the
reference renders from them, so the parity tests can compare against the reference on machines where
the reference is not available.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
import scenes  # noqa: E402
from neraulgraphics_b200 import workloads  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


def icosphere_fixture():
    wl = workloads.icosphere_worlds(worlds=16, per_world=8, seed=0)
    ref = O.Reference(wl.desc)
    ref.set_instance_transforms(wl.matrices)
    out = ref.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, normals=True, object_ids=True)
    save("icosphere_16x8_seed0", matrices=wl.matrices, cameras=wl.cameras, fov=np.float32(wl.fov), **out)


def template_fixture():
    desc = scenes.template(worlds=6)
    mats = scenes.template_matrices(6)
    cams = np.stack([scenes.camera()] * 6)
    ref = O.Reference(desc)
    ref.set_instance_transforms(mats)
    ref.set_ambient(0.1)
    out = ref.render(cams, scenes.FOV, 2, rgb=True, depth=True, normals=True, object_ids=True, frame=5)
    save("template_6w_spp2_frame5", matrices=mats, cameras=cams, fov=np.float32(scenes.FOV), ambient=np.float32(0.1),
         **out)


def body_fixture():
    """Body poses: the instance matrices are composed in single precision (the reference's GPU compose,
    restated by the oracle), then the reference renders from those matrices."""
    wl = workloads.body_worlds(worlds=16, seed=0)
    b = wl.binding
    mats = O.compose(16, 20, 20, b["body_of_instance"], b["local_pose"], b["scale"], wl.poses)
    ref = O.Reference(wl.desc)
    ref.set_instance_transforms(mats)
    out = ref.render(wl.cameras, wl.fov, 1, rgb=True, depth=True, normals=False, object_ids=True)
    rng = np.random.default_rng(5)
    origins = rng.uniform(-3, 3, size=(16, 256, 3)).astype(np.float32)
    dirs = rng.normal(size=(16, 256, 3)).astype(np.float32)
    hits = ref.cast_rays(origins, dirs, 20.0)
    save("body_16x20_seed0", poses=wl.poses, matrices=mats, cameras=wl.cameras, fov=np.float32(wl.fov),
         ray_origins=origins, ray_directions=dirs, ray_distance=hits["distance"], ray_normal=hits["normal"],
         ray_object_id=hits["object_id"], **out)


if __name__ == "__main__":
    icosphere_fixture()
    template_fixture()
    body_fixture()
