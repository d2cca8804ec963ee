"""Partial re-upload (xtgpu_scene_update): materials, samplers, textures, the
environment and the camera of a resident scene replaced without a BVH rebuild.
Every frame after an update equals, bit for bit, the frame of a scene created
from the updated description; a service sees the change after
xtgpu_service_update_scene."""
import dataclasses

import numpy as np
import pytest

from xtracer_b200 import scenes, xtgpu
from xtracer_b200.service import Service

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


def edited(spec):
    """The same geometry with other materials (textured), environment and camera."""
    tex = scenes.textured_scene("erp")
    mats = [dataclasses.replace(tex.materials[i % len(tex.materials)]) for i in range(len(spec.materials))]
    cam = scenes.Camera((1.0, 4.0, -10.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 45.0, flength=9.0, aperture=0.5)
    return dataclasses.replace(spec, materials=mats, env_type=tex.env_type, env_textures=tex.env_textures,
                               camera=cam, obj_uv_scale=np.ones((len(spec.obj_kind), 2), np.float32))


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
def test_updated_scene_renders_like_a_fresh_one(fmt):
    a = scenes.spheres_scene(64, seed=1, name="upd")
    b = edited(a)
    sc = xtgpu.Scene(a, node_formats=(fmt,))
    before, _ = sc.render(xtgpu.PATHTRACER, 48, 40, spp=4, rdepth=4, seed=3, node_format=fmt)
    sc.update(b, what=1)                       # shading only: the old camera stays
    mixed = dataclasses.replace(b, camera=a.camera)
    fresh = xtgpu.Scene(mixed, node_formats=(fmt,))
    for integ in (xtgpu.PATHTRACER, xtgpu.EMISSION):
        got, _ = sc.render(integ, 48, 40, spp=4, rdepth=4, seed=3, node_format=fmt)
        ref, _ = fresh.render(integ, 48, 40, spp=4, rdepth=4, seed=3, node_format=fmt)
        assert np.array_equal(got, ref)
    fresh.close()
    sc.update(b, what=2)                       # then the camera
    fresh = xtgpu.Scene(b, node_formats=(fmt,))
    got, _ = sc.render(xtgpu.PATHTRACER, 48, 40, spp=4, rdepth=4, seed=3, node_format=fmt)
    ref, _ = fresh.render(xtgpu.PATHTRACER, 48, 40, spp=4, rdepth=4, seed=3, node_format=fmt)
    assert np.array_equal(got, ref)
    assert not np.array_equal(got, before)
    fresh.close()
    sc.close()


def test_service_takes_the_update():
    a = scenes.spheres_scene(64, seed=1, name="upd_svc")
    b = edited(a)
    sc = xtgpu.Scene(a, node_formats=(xtgpu.NODES_W8,))
    svc = Service([sc], node_format=xtgpu.NODES_W8, use_graphs=True)
    j = svc.submit(0, xtgpu.PATHTRACER, 40, 32, 4, 4, 100.0, 5)
    svc.run()
    first = svc.result(j).copy()
    svc.release(j)
    sc.update(b)
    svc.update_scene(0)
    j = svc.submit(0, xtgpu.PATHTRACER, 40, 32, 4, 4, 100.0, 5)
    svc.run()
    got = svc.result(j).copy()
    svc.release(j)
    svc.close()
    fresh = xtgpu.Scene(b, node_formats=(xtgpu.NODES_W8,))
    ref, _ = fresh.render(xtgpu.PATHTRACER, 40, 32, spp=4, rdepth=4, seed=5, node_format=xtgpu.NODES_W8)
    fresh.close()
    sc.close()
    assert np.array_equal(got, ref)
    assert not np.array_equal(first, got)


def test_update_refuses_other_geometry():
    a = scenes.spheres_scene(16, seed=1, name="upd_bad")
    sc = xtgpu.Scene(a)
    other = scenes.spheres_scene(17, seed=1, name="upd_bad2")
    with pytest.raises(xtgpu.XtgpuError):
        sc.update(other, what=1)
    sc.close()


def test_service_after_bvh_rebuild():
    """A service's captured single-scene graphs hold the scene's node and leaf
    buffers; after a rebuild with another leaf size (new buffers) and
    xtgpu_service_update_scene, graphed waves render the rebuilt tree and
    equal xtgpu_render's frame."""
    spec = scenes.terrain_scene(20_000, seed=2, name="upd_rebuild")
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_W8,), leaf_size=1)
    svc = Service([sc], node_format=xtgpu.NODES_W8, use_graphs=True, wave_paths=1 << 14)
    j = svc.submit(0, xtgpu.PATHTRACER, 64, 48, 8, 4, 100.0, 7)
    svc.run()
    first = svc.result(j).copy()
    svc.release(j)
    sc.build_bvh(xtgpu.NODES_W8, leaf_size=3)
    svc.update_scene(0)
    for _ in range(2):
        j = svc.submit(0, xtgpu.PATHTRACER, 64, 48, 8, 4, 100.0, 7)
        svc.run()
        got = svc.result(j).copy()
        svc.release(j)
        ref, _ = sc.render(xtgpu.PATHTRACER, 64, 48, spp=8, rdepth=4, seed=7, node_format=xtgpu.NODES_W8)
        assert np.array_equal(got, ref)
        # every tree gives the same closest hits, so the frame is the first one
        assert np.array_equal(got, first)
    svc.close()
    sc.close()
