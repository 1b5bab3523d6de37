"""MuJoCo geom poses in place of instance matrices: the fused compose against the oracle's restatement of
MJWarpBatchRenderer's compose kernel (python/neraulgraphics/mujoco.py:291-302), bit for bit, and the images of
those matrices against the oracle's."""

import numpy as np
import pytest

import neraulgraphics_b200 as ng
import oracle as O
from neraulgraphics_b200 import workloads

pytestmark = pytest.mark.gpu
ALL = dict(rgb=True, depth=True, normals=True, object_ids=True)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def geom_scene(worlds=12, per_world=10, geoms=14, seed=3):
    """worlds x per_world instances carried by geoms_per_world = 14 geoms (4 of them not drawn, as a model's
    collision shapes are not), with uneven scales, random geom positions and rotation matrices."""
    rng = np.random.default_rng(seed)
    wl = workloads.icosphere_worlds(worlds=worlds, per_world=per_world, width=40, height=32, seed=seed)
    geom_of_instance = rng.permutation(geoms)[:per_world].astype(np.int32)
    scale = rng.uniform(0.4, 1.3, size=(per_world, 3)).astype(np.float32)
    xpos = (rng.uniform(-2.0, 2.0, size=(worlds, geoms, 3)) + (0.0, 0.0, -6.0)).astype(np.float32)
    q = rng.normal(size=(worlds * geoms, 4))
    xmat = np.stack([ng.make_transform((0, 0, 0), qi, 1.0).matrix[:, :3] for qi in q]).astype(np.float32)
    return wl, geom_of_instance, scale, xpos, xmat.reshape(worlds, geoms, 3, 3)


class CudaArray:
    """A foreign CUDA array (as a Warp or CuPy array is): only __cuda_array_interface__."""

    def __init__(self, t):
        self._t = t
        self.shape = tuple(t.shape)
        self.__cuda_array_interface__ = t.__cuda_array_interface__


@pytest.mark.parametrize("build", [1, 2])
def test_geom_poses_compose_and_render_as_the_oracle(torch_cuda, build):
    torch = torch_cuda
    wl, goi, scale, xpos, xmat = geom_scene()
    d = wl.desc
    want_m = O.geom_matrices(xpos, xmat, goi, scale)
    o = O.Oracle(d)
    o.set_instance_transforms(want_m)
    want = o.render(wl.cameras, 1.0, 1, **ALL, ties=True)
    for source in ("host", "torch", "foreign"):
        r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                             device="cuda:0")
        r.set_build(build)
        r.bind_geoms(goi, scale, xpos.shape[1])
        if source == "host":
            r.set_geom_poses(xpos, xmat)
        else:
            tp, tm = torch.from_numpy(xpos).cuda(), torch.from_numpy(xmat).cuda()
            r.set_geom_poses(*((tp, tm) if source == "torch" else (CudaArray(tp), CudaArray(tm))))
        got_m = r.inspect_tlas()["matrices"].reshape(want_m.shape)
        assert np.array_equal(bits(got_m), bits(want_m)), source
        got = r.render(wl.cameras, 1.0, 1, **ALL)
        ok = (want["ties"] & O.TIE_AOV_INSTANCE) == 0
        assert np.array_equal(got["object_ids"][ok], want["object_ids"][ok])
        assert np.array_equal(bits(got["depth"][ok]), bits(want["depth"][ok]))
        d_rgb = np.abs(got["rgb"].astype(int) - want["rgb"].astype(int)).max(-1)[(want["ties"] & O.TIE_RGB_INSTANCE) == 0]
        assert d_rgb.max(initial=0) <= 1


def test_geom_binding_and_poses_are_checked(torch_cuda):
    wl, goi, scale, xpos, xmat = geom_scene(worlds=4)
    d = wl.desc
    r = ng.BatchRenderer(d.width, d.height, d.world_count, 1, d.spheres, d.lights, d.floor, d.meshes, d.instances,
                         device="cuda:0")
    with pytest.raises(ValueError, match="bind_geoms"):
        r.set_geom_poses(xpos, xmat)
    bad = goi.copy()
    bad[3] = 14
    with pytest.raises(ValueError, match="instance 3 is on geom 14, but there are 14 geoms per world"):
        r.bind_geoms(bad, scale, 14)
    r.bind_geoms(goi, scale, 14)
    r.set_geom_poses(xpos, xmat)
    before = r.inspect_tlas()
    nan = xmat.copy()
    nan[2, 5, 1, 1] = np.nan
    with pytest.raises(ValueError, match="geom 33 has a NaN or infinite position or rotation"):
        r.set_geom_poses(xpos, nan)
    after = r.inspect_tlas()
    assert all(np.array_equal(before[k], after[k]) for k in before)  # a rejected input changes nothing
    with pytest.raises(ValueError, match="geom_xmat has"):
        r.set_geom_poses(xpos, xmat[:, :13])
    with pytest.raises(ValueError, match="bind_bodies"):
        r.set_body_poses(np.zeros((4, 14, 7), np.float32))
