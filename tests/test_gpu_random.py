"""The random sample distribution on the GPU (aa.cc:34-48): aa positions per
pixel at jittered offsets, each taken spp times at weight 1/(aa spp).

* With the oracle's jitter stream (keyed by seed, position and pixel) the
  GPU frame equals the oracle's up to the FP32 trace, for every camera draw
  order (pinhole, thin lens) and integrator family.
* Against the reference's frames (tests/golden/render_random.npz, libc rand()
  offsets at four seeds) the GPU's frames at four seeds of its own agree
  within the reference's noise.
* Random jobs share waves with grid jobs in the render service, render through
  the entry point that allocates nothing, record the raygraph, and bad
  distributions or levels are refused."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests import parity
from tests.parity import random_distribution_agreement
from xtracer_b200 import scenes, xtgpu
from xtracer_b200.service import Service

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RANDOM = xtgpu.SAMPLES_RANDOM
DOF = scenes.Camera((0.0, 3.0, -12.0), (0.0, 1.5, 0.0), (0.0, 1.0, 0.0), 50.0, flength=11.0, aperture=0.75)


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


def _random_case():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.random_case()


def _oracle_full(spec, code, w, h, spp, seed, aa, md=100.0, rdepth=4):
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    ys, xs = np.mgrid[0:h, 0:w]
    px = np.stack([xs.ravel(), ys.ravel()], 1)
    return orc.render(code, w, h, spp=spp, rdepth=rdepth, ao_max_distance=md, seed=seed, pixels=px, aa=aa,
                      distribution=po.SAMPLES_RANDOM)


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
@pytest.mark.parametrize("aa", [1, 4, 7])
def test_random_same_stream_as_oracle(aa, fmt):
    """Stencil coverage equals the oracle's on all but edge-grazing pixels and
    depth is within 1e-5 relative; the rays traced are aa x spp per pixel."""
    cam, w, h, spp, _, _ = _random_case()
    spec = scenes.spheres_scene(64, seed=1, name="rnd_same", camera=cam)
    sc = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    for code in (xtgpu.STENCIL, xtgpu.DEPTH):
        img, rays = sc.render(code, w, h, spp=spp, seed=17, node_format=fmt, aa=aa, distribution=RANDOM)
        o, orays = _oracle_full(spec, code, w, h, spp, 17, aa)
        assert rays == orays == w * h * aa * spp
        got = img.reshape(-1, 4)
        if code == xtgpu.STENCIL:
            assert (got == o).all(axis=1).mean() >= 0.998, (got != o).any(axis=1).sum()
        else:
            rel = np.abs(got[:, 0] - o[:, 0]) / np.maximum(np.abs(o[:, 0]), 1e-6)
            assert np.mean(rel <= 1e-5) >= 0.99, np.sort(rel)[-5:]
    sc.close()


@pytest.mark.parametrize("cam, w, h", [
    (scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_ERP, orientation=(0.25, -0.5, 0.125)), 64, 32),
    (scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_ODS, orientation=(0.0, 0.75, 0.0), ipd=0.125), 48, 48),
    (scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_CUBEMAP), 16, 96)], ids=["erp", "ods", "cubemap"])
def test_random_through_every_camera_same_stream_as_oracle(cam, w, h):
    """The jittered positions feed the equirectangular, omni-directional stereo
    and cubemap cameras as they feed the pinhole one: stencil equal to the
    oracle's, depth within 1e-5 relative in the hit distance (|d depth| <=
    1e-5 |depth| max(1, |depth|), depth being 1/log t)."""
    spec = scenes.spheres_scene(64, seed=1, name="rnd_cam", camera=cam)
    sc = xtgpu.Scene(spec)
    for code in (xtgpu.STENCIL, xtgpu.DEPTH):
        img, rays = sc.render(code, w, h, spp=2, seed=23, aa=3, distribution=RANDOM)
        o, orays = _oracle_full(spec, code, w, h, 2, 23, 3)
        assert rays == orays == w * h * 6
        got = img.reshape(-1, 4)
        if code == xtgpu.STENCIL:
            assert (got == o).all(axis=1).mean() >= 0.998, (got != o).any(axis=1).sum()
        else:
            D = np.abs(o[:, 0].astype(np.float64))
            rel = np.abs(got[:, 0] - o[:, 0]) / np.maximum(D, 1e-6)
            assert np.mean(rel <= 1e-5 * np.maximum(1.0, D)) >= 0.99, np.sort(rel)[-5:]
    sc.close()


def test_random_with_lens_and_ao_same_stream_as_oracle():
    """The jitter comes from a stream of its own, so the thin-lens draws and
    AO's hemisphere draws keep their places on the sample's stream."""
    spec = scenes.spheres_scene(64, seed=1, name="rnd_dof", camera=DOF)
    w, h = 40, 40
    sc = xtgpu.Scene(spec)
    img, rays = sc.render(xtgpu.DEPTH, w, h, spp=2, seed=41, aa=3, distribution=RANDOM)
    o, orays = _oracle_full(spec, po.DEPTH, w, h, 2, 41, 3)
    assert rays == orays == w * h * 6
    rel = np.abs(img.reshape(-1, 4)[:, 0] - o[:, 0]) / np.maximum(np.abs(o[:, 0]), 1e-6)
    assert np.mean(rel <= 1e-5) >= 0.99, np.sort(rel)[-5:]
    img, rays = sc.render(xtgpu.AO, w, h, spp=4, seed=43, ao_max_distance=0.5, aa=2, distribution=RANDOM)
    o, orays = _oracle_full(spec, po.AO, w, h, 4, 43, 2, md=0.5)
    o2, _ = _oracle_full(spec, po.AO, w, h, 4, 44, 2, md=0.5)
    parity.same_stream_bar(img, o, o2, "random aa2 dof ao")
    assert abs(rays - orays) <= 0.01 * orays
    sc.close()


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
def test_random_frames_within_reference_noise(fmt):
    """Stencil (aa 1 and 4) and depth (aa 4) frames at four seeds against the
    reference's four: equal ray counts, the same coverage values, and frame and
    per-pixel means within the noise of the seeds."""
    cam, w, h, spp, cases, seeds = _random_case()
    g = np.load(os.path.join(GOLD, "render_random.npz"))
    sc = xtgpu.Scene(scenes.spheres_scene(64, seed=1, name="cam_random", camera=cam), node_formats=(fmt,),
                     leaf_size=1)
    for integ, aa in cases:
        key = "%s_aa%d" % (integ, aa)
        code = xtgpu.STENCIL if integ == "stencil" else xtgpu.DEPTH
        xy = g[key + "_xy"]
        O = []
        for s, ref_rays in zip((1001, 1002, 1003, 1004), g[key + "_rays"]):
            img, rays = sc.render(code, w, h, spp=spp, seed=s, node_format=fmt, aa=aa, distribution=RANDOM)
            assert rays == int(ref_rays)
            O.append(img[xy[:, 1], xy[:, 0]])
        random_distribution_agreement(g[key + "_rgba"], np.stack(O), 3 if integ == "stencil" else 0,
                                      aa if integ == "stencil" else None)
    sc.close()


def test_random_and_grid_jobs_in_the_mix_equal_alone():
    """Random and grid jobs of several scenes share waves; each frame equals
    the scene's own render."""
    cam, _, _, _, _, _ = _random_case()
    res = [xtgpu.Scene(scenes.spheres_scene(64, seed=1, name="rmix0", camera=cam)),
           xtgpu.Scene(scenes.spheres_scene(64, seed=1, name="rmix1", camera=DOF))]
    jobs = [(0, xtgpu.DEPTH, 48, 40, 2, 4, RANDOM, 1), (1, xtgpu.AO, 40, 40, 2, 3, RANDOM, 2),
            (0, xtgpu.STENCIL, 32, 32, 1, 2, xtgpu.SAMPLES_GRID, 3), (1, xtgpu.PATHTRACER, 32, 32, 4, 5, RANDOM, 4),
            (0, xtgpu.NORMAL, 24, 24, 2, 1, RANDOM, 5)]
    alone = [res[s].render(integ, w, h, spp=spp, rdepth=4, ao_max_distance=0.5, seed=seed, aa=aa, distribution=dist)
             for (s, integ, w, h, spp, aa, dist, seed) in jobs]
    for wave in (1 << 22, 777):
        svc = Service(res, wave_paths=wave, use_graphs=True, merge_jobs=True, memory_budget=1 << 30)
        ids = [svc.submit(s, integ, w, h, spp, 4, 0.5, seed, aa=aa, distribution=dist)
               for (s, integ, w, h, spp, aa, dist, seed) in jobs]
        svc.run()
        for jid, (ref, rays) in zip(ids, alone):
            assert svc.poll(jid).state == 2
            assert svc.poll(jid).rays == rays
            assert np.array_equal(svc.result(jid), ref, equal_nan=True), "job %d (wave %d)" % (jid, wave)
            svc.release(jid)
        svc.close()
    for r in res:
        r.close()


def test_noalloc_tile_with_random_equals_render():
    import torch
    spec = scenes.spheres_scene(64, seed=1, name="na_rnd", camera=DOF)
    sc = xtgpu.Scene(spec)
    rect = (8, 8, 24, 24)
    ref, ref_rays = sc.render(xtgpu.AO, 32, 32, spp=4, ao_max_distance=0.5, seed=5, rect=rect, aa=5,
                              distribution=RANDOM)
    out = torch.empty((16, 16, 4), dtype=torch.float32, device="cuda")
    p = xtgpu.RenderParams(xtgpu.AO, 32, 32, 4, 4, 0.5, 5, xtgpu.NODES_FP32, *rect, 5, RANDOM)
    rays = C.c_uint64()
    st = xtgpu.lib().xtgpu_render_tile_noalloc(sc.handle, C.byref(p), C.c_void_p(out.data_ptr()), C.byref(rays),
                                               None)
    assert st == 0, xtgpu.lib().xtgpu_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    assert int(rays.value) == ref_rays
    sc.close()


def test_random_raygraph_follows_oracle():
    """The raygraph of a random-distribution depth render holds aa x spp records
    per pixel; their origins, hit points and running colours follow the
    oracle's, and the frame equals the plain render."""
    cam, _, _, _, _, _ = _random_case()
    spec = scenes.spheres_scene(64, seed=1, name="rnd_rg", camera=cam)
    w, h, spp, aa = 40, 36, 2, 3
    sc = xtgpu.Scene(spec)
    frame, rec = sc.render_raygraph(w, h, spp=spp, aa=aa, distribution=RANDOM)
    plain, _ = sc.render(xtgpu.DEPTH, w, h, spp=spp, rdepth=1, aa=aa, distribution=RANDOM)
    sc.close()
    assert rec.shape == (w * h * aa * spp, 10)
    assert np.array_equal(frame, plain)
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    oframe, orec = orc.render_raygraph(w, h, spp=spp, aa=aa, pixels=po.raygraph_pixel_order(w, h),
                                       distribution=po.SAMPLES_RANDOM)
    assert orec.shape == rec.shape
    assert np.allclose(rec[:, :3], orec[:, :3], atol=1e-5)
    hit_g, hit_o = np.abs(rec[:, 3:6]).sum(1) > 0, np.abs(orec[:, 3:6]).sum(1) > 0
    assert np.mean(hit_g == hit_o) >= 0.998
    both = hit_g & hit_o
    d = np.abs(rec[both, 3:6] - orec[both, 3:6]).max(1)
    assert np.mean(d <= 1e-3 * np.maximum(1.0, np.abs(orec[both, 3:6]).max(1))) >= 0.995, np.sort(d)[-5:]


def test_bad_distributions_and_levels_are_refused():
    sc = xtgpu.Scene(scenes.spheres_scene(16, seed=1, name="rnd_bad"))
    for aa, dist in ((2, 2), (2, -1), (257, RANDOM), (-1, RANDOM), (17, xtgpu.SAMPLES_GRID)):
        with pytest.raises(xtgpu.XtgpuError):
            sc.render(xtgpu.STENCIL, 8, 8, spp=1, aa=aa, distribution=dist)
    img, rays = sc.render(xtgpu.STENCIL, 4, 4, spp=1, aa=256, distribution=RANDOM)   # 256 jittered positions
    assert rays == 4 * 4 * 256
    img, rays = sc.render(xtgpu.STENCIL, 4, 4, spp=1, aa=0, distribution=RANDOM)     # level 0 renders as 1
    assert rays == 4 * 4
    with pytest.raises(xtgpu.XtgpuError):
        sc.render(xtgpu.STENCIL, 4, 4, spp=1 << 24, aa=256, distribution=RANDOM)     # 2^32 samples per pixel
    for aa, dist in ((17, xtgpu.SAMPLES_GRID), (257, RANDOM), (1, 2)):   # refused before any buffer is sized
        with pytest.raises(xtgpu.XtgpuError):
            sc.render_raygraph(8, 8, spp=1, aa=aa, distribution=dist)
    svc = Service([sc], wave_paths=1 << 16)
    with pytest.raises(xtgpu.XtgpuError):
        svc.submit(0, xtgpu.STENCIL, 8, 8, 1, aa=2, distribution=3)
    svc.close()
    sc.close()
