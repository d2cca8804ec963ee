"""Degenerate inputs on the GPU, against the oracle: a scene of one plane and
no primitive for any tree to hold, a scene with no object at all (every ray
meets the environment), and one-pixel frames and rectangles; every node
format."""
import dataclasses

import numpy as np
import pytest

from oracle import pyoracle as po
from tests import parity
from xtracer_b200 import scenes, xtgpu

pytestmark = pytest.mark.gpu
FORMATS = (xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8)


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


def plane_only():
    return scenes.spheres_scene(0, seed=1, name="planeonly", with_light=False)


def empty():
    sp = plane_only()
    return dataclasses.replace(sp, name="empty", planes=np.zeros((0, 4), np.float32),
                               obj_kind=np.zeros(0, np.int32), obj_first=np.zeros(0, np.int32),
                               obj_count=np.zeros(0, np.int32), obj_material=np.zeros(0, np.int32))


def _all_px(w, h):
    ys, xs = np.mgrid[0:h, 0:w]
    return np.stack([xs.ravel(), ys.ravel()], 1)


@pytest.mark.parametrize("make", [plane_only, empty])
@pytest.mark.parametrize("fmt", FORMATS)
def test_scenes_without_primitives(make, fmt):
    spec = make()
    w, h = 40, 30
    sc = xtgpu.Scene(spec, node_formats=(fmt,))
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    px = _all_px(w, h)
    for integ, code in ((xtgpu.STENCIL, po.STENCIL), (xtgpu.DEPTH, po.DEPTH)):
        g, rays = sc.render(integ, w, h, spp=2, node_format=fmt)
        o, orays = orc.render(code, w, h, spp=2, pixels=px)
        assert rays == orays == w * h * 2
        g = g.reshape(-1, 4).astype(np.float64)
        if integ == xtgpu.STENCIL:
            assert np.array_equal(g, o)
        else:
            hit = o[:, 0] != 0
            assert np.array_equal(g[~hit], o[~hit])
            if hit.any():
                assert np.abs(1.0 / g[hit, 0] - 1.0 / o[hit, 0]).max() <= 1e-5
    # pathtracer on the same stream: the plane is the only thing a path can meet
    g, rays = sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=3, node_format=fmt)
    o, orays = orc.render(po.PATHTRACER, w, h, spp=8, rdepth=4, seed=3, pixels=px)
    o2, _ = orc.render(po.PATHTRACER, w, h, spp=8, rdepth=4, seed=4, pixels=px)
    assert abs(rays - orays) <= 0.01 * orays
    if make is empty:
        # every path misses at once: the environment in the camera ray's direction
        assert rays == w * h * 8
        assert np.allclose(g.reshape(-1, 4), o, rtol=1e-5, atol=1e-6)
    else:
        parity.same_stream_bar(g, o, o2, "%s pt fmt %d" % (spec.name, fmt))
    sc.close()


@pytest.mark.parametrize("fmt", FORMATS)
def test_one_pixel_frames_and_rectangles(fmt):
    spec = scenes.spheres_scene(64, seed=1, name="onepx")
    sc = xtgpu.Scene(spec, node_formats=(fmt,))
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    g, rays = sc.render(xtgpu.DEPTH, 1, 1, spp=3, node_format=fmt)
    o, _ = orc.render(po.DEPTH, 1, 1, spp=3, pixels=np.array([[0, 0]]))
    assert rays == 3 and g.shape == (1, 1, 4)
    assert np.allclose(g.reshape(-1, 4), o, rtol=1e-5, atol=0)
    full, _ = sc.render(xtgpu.PATHTRACER, 33, 17, spp=4, rdepth=4, seed=9, node_format=fmt)
    for (x, y) in ((0, 0), (32, 16), (17, 5)):
        one, r1 = sc.render(xtgpu.PATHTRACER, 33, 17, spp=4, rdepth=4, seed=9, node_format=fmt,
                            rect=(x, y, x + 1, y + 1))
        assert one.shape == (1, 1, 4)
        assert np.array_equal(one[0, 0], full[y, x])
    sc.close()
