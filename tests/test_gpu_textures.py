"""Material and environment samplers on the GPU (sampler_*.cc): 2D textures
with nearest and bilinear filtering, ERP, cubemap and gradient samplers on
diffuse, specular and emissive, ERP and cubemap environments.

* Emission (aa 2) and depth-1 pathtracer frames are deterministic: against the
  reference's own renders of the same .scn and PNG files.  The texcoord is
  formed from the FP32 hit, so continuous samplers (bilinear, gradient) move
  by a few float ulps (1e-5); a texcoord on the other side of a texel edge
  than the reference's would take the neighbouring texel (0.1 % allowed).
* Depth-4 paths: with the oracle's random stream, path by path; with its own,
  within the reference's noise.
* Textured jobs render to the same bits alone and in a service mix."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests import parity
from xtracer_b200 import scenes, xtgpu
from xtracer_b200.service import Service

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
W, H = 64, 48   # the frame size of render_textures.npz


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_frames_vs_reference_golden(env, fmt):
    g = np.load(os.path.join(GOLD, "render_textures.npz"))
    spec = scenes.textured_scene(env)
    sc = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    for integ, code, spp, rdepth, aa in (("emission", xtgpu.EMISSION, 2, 1, 2),
                                         ("pathtracer", xtgpu.PATHTRACER, 2, 1, 1)):
        img, rays = sc.render(code, W, H, spp=spp, rdepth=rdepth, node_format=fmt, aa=aa)
        assert rays == int(g["%s_%s_rays" % (env, integ)])
        xy = g["%s_%s_xy" % (env, integ)]
        got = img[xy[:, 1], xy[:, 0]]
        ref = g["%s_%s_rgba" % (env, integ)]
        # nearest lookups land on the reference's texel; bilinear and gradient
        # samples move with the FP32 texcoord by a few float ulps
        d = np.abs(got - ref).max(axis=1)
        assert np.mean(d <= 1e-5) >= 0.999, (env, integ, np.sort(d)[-5:])
        assert np.mean(d == 0) >= 0.9, (env, integ, np.mean(d == 0))
    sc.close()


def _oracle_full(spec, code, spp, seed, rdepth=4):
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    ys, xs = np.mgrid[0:H, 0:W]
    px = np.stack([xs.ravel(), ys.ravel()], 1)
    return orc.render(code, W, H, spp=spp, rdepth=rdepth, seed=seed, pixels=px)


@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_pathtracer_same_stream_as_oracle(env):
    """Textured diffuse, specular and emissive samples along depth-4 paths:
    GPU (FP32 trace) and oracle (FP64) on the same random stream differ only
    where a rounding difference sends a path another way."""
    spec = scenes.textured_scene(env)
    sc = xtgpu.Scene(spec)
    img, rays = sc.render(xtgpu.PATHTRACER, W, H, spp=8, rdepth=4, seed=61)
    sc.close()
    o, orays = _oracle_full(spec, po.PATHTRACER, 8, 61)
    o2, _ = _oracle_full(spec, po.PATHTRACER, 8, 62)
    parity.same_stream_bar(img, o, o2, "textured %s pt" % env)
    assert abs(rays - orays) <= 0.01 * orays


def _truth(name):
    t = np.load(os.path.join(GOLD, "truth.npz"))
    return t[name + "_xy"], t[name + "_rgba"]


@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_pathtracer_within_reference_noise(env):
    """Per-pixel RMSE against the 4096-spp render within the reference's own
    at 16 spp (four reference seeds)."""
    g = np.load(os.path.join(GOLD, "render_textures.npz"))
    spec = scenes.textured_scene(env)
    xy, truth = _truth("textures_%s_pt" % env)
    assert np.array_equal(xy, g["%s_pt_xy" % env])
    sc = xtgpu.Scene(spec)
    frames = []
    for seed in (777, 778):
        img, _ = sc.render(xtgpu.PATHTRACER, W, H, spp=16, rdepth=4, seed=seed)
        frames.append(img[xy[:, 1], xy[:, 0]])
    sc.close()
    R = g["%s_pt_rgba" % env]
    parity.converged_rmse_bar(np.stack(frames), truth, [parity.rmse(r, truth) for r in R], "textured %s" % env)


def test_textured_jobs_alone_equal_jobs_in_the_mix():
    res = [xtgpu.Scene(scenes.textured_scene("erp")), xtgpu.Scene(scenes.textured_scene("cubemap")),
           xtgpu.Scene(scenes.spheres_scene(64, seed=1, name="plain64"))]
    jobs = [(0, xtgpu.PATHTRACER, 64, 48, 4, 1, 1), (1, xtgpu.EMISSION, 40, 30, 2, 2, 2),
            (2, xtgpu.PATHTRACER, 32, 32, 4, 1, 3), (1, xtgpu.PATHTRACER, 48, 48, 2, 1, 4)]
    alone = [res[s].render(integ, w, h, spp=spp, rdepth=4, seed=seed, aa=aa)
             for (s, integ, w, h, spp, aa, seed) in jobs]
    svc = Service(res, wave_paths=1500, use_graphs=True, merge_jobs=True, memory_budget=1 << 30)
    ids = [svc.submit(s, integ, w, h, spp, 4, 100.0, seed, aa=aa) for (s, integ, w, h, spp, aa, seed) in jobs]
    svc.run()
    for jid, (ref, rays) in zip(ids, alone):
        assert svc.poll(jid).state == 2 and svc.poll(jid).rays == rays
        assert np.array_equal(svc.result(jid), ref), "job %d" % jid
        svc.release(jid)
    svc.close()
    for r in res:
        r.close()


def test_obj_mtl_frames_vs_reference_golden():
    """Meshes loaded from an OBJ with an MTL library (BlinnPhong with Kd / Ks or
    map_Kd / map_Ks, Emissive with Ke or map_Ke, textures flipped
    horizontally): against the reference's frames of the same files."""
    g = np.load(os.path.join(GOLD, "render_mtl.npz"))
    sc = xtgpu.Scene(scenes.mtl_scene())
    for integ, code in (("depth", xtgpu.DEPTH), ("uv", xtgpu.UV), ("emission", xtgpu.EMISSION),
                        ("pathtracer", xtgpu.PATHTRACER)):
        img, rays = sc.render(code, 64, 48, spp=2, rdepth=1)
        assert rays == int(g["%s_rays" % integ])
        xy = g["%s_xy" % integ]
        got, ref = img[xy[:, 1], xy[:, 0]], g["%s_rgba" % integ]
        d = np.abs(got - ref).max(axis=1)
        if integ == "depth":   # 1/log(t): 1e-5 relative in t
            D = np.abs(ref[:, 0].astype(np.float64))
            assert np.mean(d <= 1e-5 * D * np.maximum(1.0, D) + 1e-7) >= 0.998, np.sort(d)[-5:]
        elif integ == "uv":    # texcoords from the FP32 hit
            assert np.mean(d <= 1e-4) >= 0.998, np.sort(d)[-5:]
        else:
            assert np.mean(d <= 1e-5) >= 0.998, (integ, np.sort(d)[-5:])
    xy, truth = _truth("mtl_pt")
    assert np.array_equal(xy, g["pt_xy"])
    frames = []
    for seed in (777, 778):
        img, _ = sc.render(xtgpu.PATHTRACER, 64, 48, spp=16, rdepth=4, seed=seed)
        frames.append(img[xy[:, 1], xy[:, 0]])
    sc.close()
    parity.converged_rmse_bar(np.stack(frames), truth, [parity.rmse(r, truth) for r in g["pt_rgba"]], "mtl pt")
