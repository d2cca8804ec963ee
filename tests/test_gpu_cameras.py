"""Cameras and grid anti-aliasing on the GPU (camera/*.cc, aa.cc): thin-lens
perspective with depth of field, equirectangular, omni-directional stereo and
cubemap cameras, aa^2 grid positions per pixel.

* Stencil, depth and normal frames through each camera, with aa 2 or 3,
  against the reference's own renders (tests/golden/render_cameras.npz).
* Depth of field: the lens draws come first on each sample's random stream,
  so with the oracle's stream the GPU frame equals the oracle's up to FP32
  rounding; with its own stream it lies within the reference's noise.
* aa through the render service (alone = in the mix) and the entry point that
  allocates nothing; out-of-range aa and cubemap heights are refused."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests import parity
from xtracer_b200 import scenes, xtgpu
from xtracer_b200.service import Service

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CODES = {"stencil": xtgpu.STENCIL, "depth": xtgpu.DEPTH, "normal": xtgpu.NORMAL}
DOF = scenes.Camera((0.0, 3.0, -12.0), (0.0, 1.5, 0.0), (0.0, 1.0, 0.0), 50.0, flength=11.0, aperture=0.75)


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


def _camera_cases():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.camera_cases()


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
@pytest.mark.parametrize("case", range(4))
def test_camera_frames_vs_reference_golden(case, fmt):
    """Per camera: the rays traced are aa^2 x spp per pixel; stencil equals the
    reference's frame and normal is within 1e-4 on all but grazing pixels (the
    GPU traces the FP64 camera ray in FP32).  Depth is 1/log(t), whose
    relative error is the hit distance's times |depth|; the ERP, ODS and
    cubemap cameras sit among the spheres, where t near 1 gives depths in the
    thousands, so the bound is 1e-5 relative in t: |d depth| <= 1e-5 |depth|
    max(1, |depth|)."""
    g = np.load(os.path.join(GOLD, "render_cameras.npz"))
    tag, cam, w, h, aa = _camera_cases()[case]
    spec = scenes.spheres_scene(64, seed=1, name="cam_" + tag, camera=cam)
    sc = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    for integ, code in CODES.items():
        img, rays = sc.render(code, w, h, spp=2, seed=1, node_format=fmt, aa=aa)
        assert rays == int(g["%s_%s_rays" % (tag, integ)]) == w * h * aa * aa * 2
        xy = g["%s_%s_xy" % (tag, integ)]
        got = img[xy[:, 1], xy[:, 0]]
        ref = g["%s_%s_rgba" % (tag, integ)]
        if integ == "stencil":
            assert (got == ref).all(axis=1).mean() >= 0.998, (tag, (got != ref).any(axis=1).sum())
        elif integ == "depth":
            D = np.abs(ref[:, 0].astype(np.float64))
            rel = np.abs(got[:, 0] - ref[:, 0]) / np.maximum(D, 1e-6)
            assert np.mean(rel <= 1e-5 * np.maximum(1.0, D)) >= 0.998, (tag, np.sort(rel)[-5:])
            assert (got[:, 3] == ref[:, 3]).all()
        else:
            nan_g, nan_r = np.isnan(got).any(axis=1), np.isnan(ref).any(axis=1)
            assert np.mean(nan_g == nan_r) >= 0.999
            both = ~nan_g & ~nan_r
            d = np.abs(got[both] - ref[both]).max(axis=1)
            assert np.mean(d <= 1e-4) >= 0.99, (tag, np.sort(d)[-5:])
    sc.close()


def _oracle_full(spec, code, w, h, spp, seed, aa=1, md=100.0, rdepth=4):
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    ys, xs = np.mgrid[0:h, 0:w]
    px = np.stack([xs.ravel(), ys.ravel()], 1)
    return orc.render(code, w, h, spp=spp, rdepth=rdepth, ao_max_distance=md, seed=seed, pixels=px, aa=aa)


def test_depth_of_field_same_stream_as_oracle():
    """The two lens draws are the first values of the sample's stream (the
    oracle's order), so the thin-lens rays and the depth frame follow the
    oracle's up to the FP32 trace."""
    spec = scenes.spheres_scene(64, seed=1, name="dof", camera=DOF)
    w, h = 48, 48
    sc = xtgpu.Scene(spec)
    img, rays = sc.render(xtgpu.DEPTH, w, h, spp=4, seed=41, aa=2)
    sc.close()
    o, orays = _oracle_full(spec, po.DEPTH, w, h, 4, 41, aa=2)
    assert rays == orays == w * h * 16
    got = img.reshape(-1, 4)
    rel = np.abs(got[:, 0] - o[:, 0]) / np.maximum(np.abs(o[:, 0]), 1e-6)
    print("[dof depth] %.4f of pixels within 1e-5 of the oracle (16 rays each)" % np.mean(rel <= 1e-5))
    assert np.mean(rel <= 1e-5) >= 0.99, np.sort(rel)[-5:]


def test_ao_after_lens_draws_same_stream_as_oracle():
    """AO's hemisphere draws continue the stream after the two lens draws."""
    spec = scenes.spheres_scene(64, seed=1, name="dofao", camera=DOF)
    w, h = 40, 40
    sc = xtgpu.Scene(spec)
    img, rays = sc.render(xtgpu.AO, w, h, spp=8, seed=43, ao_max_distance=0.5)
    sc.close()
    o, orays = _oracle_full(spec, po.AO, w, h, 8, 43, md=0.5)
    o2, _ = _oracle_full(spec, po.AO, w, h, 8, 44, md=0.5)
    parity.same_stream_bar(img, o, o2, "dof ao")
    assert abs(rays - orays) <= 0.01 * orays


def test_depth_of_field_within_reference_noise():
    """The reference draws its lens offsets from the C library's rand(); its
    depth frames at four seeds (31-34) give its noise at 16 spp.  The GPU's
    frames, from their own stream, have per-pixel RMSE against the 4096-spp
    render within that noise."""
    g = np.load(os.path.join(GOLD, "render_cameras.npz"))
    t = np.load(os.path.join(GOLD, "truth.npz"))
    xy, truth = t["dof_depth_xy"], t["dof_depth_rgba"]
    assert np.array_equal(xy, g["dof_depth_xy"])
    spec = scenes.spheres_scene(64, seed=1, name="cam_dof", camera=DOF)
    sc = xtgpu.Scene(spec)
    frames = []
    for seed in (777, 778):
        img, _ = sc.render(xtgpu.DEPTH, 48, 48, spp=16, seed=seed)
        frames.append(img[xy[:, 1], xy[:, 0]])
    sc.close()
    parity.converged_rmse_bar(np.stack(frames), truth, [parity.rmse(r, truth) for r in g["dof_depth_rgba"]],
                              "dof depth")


def test_aa_jobs_alone_equal_jobs_in_the_mix():
    """Jobs of scenes with different cameras and aa levels share waves; each
    frame equals the scene's own render."""
    cams = [c for _, c, _, _, _ in _camera_cases()] + [DOF]
    res = [xtgpu.Scene(scenes.spheres_scene(64, seed=1, name="mix%d" % i, camera=c)) for i, c in enumerate(cams)]
    jobs = [(0, xtgpu.DEPTH, 48, 40, 2, 3, 1), (1, xtgpu.AO, 96, 48, 2, 2, 2), (2, xtgpu.STENCIL, 64, 64, 1, 2, 3),
            (3, xtgpu.NORMAL, 24, 144, 2, 2, 4), (4, xtgpu.PATHTRACER, 40, 40, 4, 1, 5),
            (4, xtgpu.DEPTH, 32, 32, 2, 2, 6)]
    alone = [res[s].render(integ, w, h, spp=spp, rdepth=4, ao_max_distance=0.5, seed=seed, aa=aa)
             for (s, integ, w, h, spp, aa, seed) in jobs]
    for wave in (1 << 22, 999):
        svc = Service(res, wave_paths=wave, use_graphs=True, merge_jobs=True, memory_budget=1 << 30)
        ids = [svc.submit(s, integ, w, h, spp, 4, 0.5, seed, aa=aa) for (s, integ, w, h, spp, aa, seed) in jobs]
        svc.run()
        for jid, (ref, rays) in zip(ids, alone):
            assert svc.poll(jid).state == 2
            assert svc.poll(jid).rays == rays
            assert np.array_equal(svc.result(jid), ref, equal_nan=True), "job %d (wave %d)" % (jid, wave)
            svc.release(jid)
        svc.close()
    for r in res:
        r.close()


def test_noalloc_tile_with_aa_equals_render():
    import torch
    spec = scenes.spheres_scene(64, seed=1, name="na_aa", camera=DOF)
    sc = xtgpu.Scene(spec)
    rect = (8, 8, 24, 24)
    ref, ref_rays = sc.render(xtgpu.AO, 32, 32, spp=4, ao_max_distance=0.5, seed=5, rect=rect, aa=3)
    out = torch.empty((16, 16, 4), dtype=torch.float32, device="cuda")
    p = xtgpu.RenderParams(xtgpu.AO, 32, 32, 4, 4, 0.5, 5, xtgpu.NODES_FP32, *rect, 3)
    rays = C.c_uint64()
    st = xtgpu.lib().xtgpu_render_tile_noalloc(sc.handle, C.byref(p), C.c_void_p(out.data_ptr()), C.byref(rays),
                                               None)
    assert st == 0, xtgpu.lib().xtgpu_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    assert int(rays.value) == ref_rays
    sc.close()


def test_bad_aa_and_cubemap_heights_are_refused():
    sc = xtgpu.Scene(scenes.spheres_scene(16, seed=1, name="cube",
                                          camera=scenes.Camera((0.0, 1.0, 0.0), type=scenes.CAM_CUBEMAP)))
    for w, h, aa in ((24, 100, 1), (24, 5, 1), (24, 144, 17), (24, 144, -1)):
        with pytest.raises(xtgpu.XtgpuError):
            sc.render(xtgpu.STENCIL, w, h, spp=1, aa=aa)
    img, rays = sc.render(xtgpu.STENCIL, 24, 144, spp=1, aa=0)   # 0 = the pixel centre
    assert rays == 24 * 144
    sc.close()
