"""Parity at the full sizes of the benchmark configurations.

* Pathtracer, 64 spheres + plane, 256x256, 16 spp, depth 4: per-pixel RMSE
  against a 4096-spp render made on the CPU by the oracle (truth.npz) within
  the reference renderer's own RMSE at 16 spp (four reference seeds, rendered
  by XTracer's code when the fixture was made).
* Depth + stencil, 999,698-triangle terrain, 1920x1080, 1 spp: primary hits on
  every 8th pixel in x and y against the FP64 oracle (>= 99.99 % agreement,
  every disagreement a tie or a grazing hit), and on every pixel where the
  primitive agrees the stencil equal and the hit distance within 1e-5
  relative; the Q8 and W8 frames equal to the FP32 frames.
* AO, 2M-triangle hairball, 1024x1024, 64 spp, distance 0.2: per-pixel RMSE
  on a 32x32 lattice against a 4096-spp oracle render within the equal-spp
  noise, and against the oracle on the same random stream (the divergence
  below a quarter of the noise); Q8 and W8 frames equal to FP32.
* Precision scene, 8M triangles, Phong/Blinn-Phong, sphere and mesh lights:
  primary hits of FP32, Q8 and W8 nodes against the FP64 oracle on every 8th
  pixel; a 64x64 crop at 16 spp, depth 8, against a 4096-spp oracle render
  within the equal-spp noise and against the oracle on the same stream; the
  1920x1080, 256-spp, depth-8 frame with Q8 and W8 nodes equal to the one
  with FP32 nodes (hence equal RMSE).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests import parity
from xtracer_b200 import scenes, xtgpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


def lattice(w, h, step):
    ys, xs = np.mgrid[step // 2:h:step, step // 2:w:step]
    return np.stack([xs.ravel(), ys.ravel()], 1)


def hits_vs_oracle(spec, sc, orc, w, h, px, fmt):
    """Primary hits of the GPU (C ABI trace of the FP64 camera rays rounded to
    FP32) against the oracle on the pixels px; returns (agreement fraction,
    max relative t error where both hit the same primitive)."""
    org, dirs = po.camera_rays(spec, w, h, px)
    g = sc.intersection(org.astype(np.float32), dirs.astype(np.float32), node_format=fmt)
    r = orc.trace(org, dirs)
    r_gid = parity.oracle_global_prim(spec, r["obj"], r["prim"])
    g_hit = (g["prim"] != 0xffffffff).astype(np.int32)
    g_gid = g["prim"].astype(np.int64)
    n_agree, tie, graze, bad = parity.classify(spec, org, dirs, g_hit, g_gid, g["t"].astype(np.float64),
                                               r["hit"], r_gid, r["t"])
    assert not bad, "unexplained disagreements at %s" % bad[:10]
    m = (g_hit == 1) & (r["hit"] == 1) & (g_gid == r_gid)
    rel = np.abs(g["t"][m].astype(np.float64) - r["t"][m]) / r["t"][m]
    return n_agree / g_hit.size, float(rel.max()) if rel.size else 0.0


def _truth(name):
    import os
    t = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "truth.npz"))
    return {k[len(name) + 1:]: t[k] for k in t.files if k.startswith(name + "_")}


def test_config_pathtracer_spheres_rmse_within_reference_noise():
    """The north star's bar at config 1's size: RMSE against the 4096-spp
    render within the reference's own at equal spp."""
    spec = scenes.spheres_scene(64, seed=1)
    w = h = 256
    T = _truth("config1")
    xy = T["xy"]
    sc = xtgpu.Scene(spec)
    frames, rays = [], []
    for seed in (1, 2):
        img, r = sc.render(xtgpu.PATHTRACER, w, h, spp=16, rdepth=4, seed=seed)
        frames.append(img[xy[:, 1], xy[:, 0]])
        rays.append(r)
    sc.close()
    parity.converged_rmse_bar(np.stack(frames), T["rgba"], T["ref_rmse"], "config1 pt 256x256 16spp")
    # the reference's frame means at 16 spp bracket the GPU's within their spread
    gm = np.mean([f[:, :3].astype(np.float64).mean(0) for f in frames], axis=0)
    rm = T["ref_mean"]
    assert np.all(np.abs(gm - rm.mean(0)) <= 5 * rm.std(0, ddof=1) + 1e-4), (gm, rm)


def test_config_terrain_1m_depth_stencil_full_hd():
    spec = scenes.terrain_scene(999_698, seed=2)
    w, h = 1920, 1080
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8))
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    px = lattice(w, h, 8)   # 240 x 135 = 32,400 rays
    for fmt in (xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8):
        agree, rel = hits_vs_oracle(spec, sc, orc, w, h, px, fmt)
        assert agree >= 0.9999 and rel <= 1e-5, (fmt, agree, rel)
    frames = {}
    for fmt in (xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8):
        for integ in (xtgpu.STENCIL, xtgpu.DEPTH):
            img, rays = sc.render(integ, w, h, spp=1, node_format=fmt)
            assert rays == w * h
            frames[fmt, integ] = img
    for integ in (xtgpu.STENCIL, xtgpu.DEPTH):
        for fmt in (xtgpu.NODES_Q8, xtgpu.NODES_W8):
            same = np.all(frames[xtgpu.NODES_FP32, integ] == frames[fmt, integ], axis=2)
            assert same.mean() >= 0.9999, (integ, fmt, same.mean())
    # stencil and depth on the lattice against the oracle's integrators,
    # pixel by pixel where the primitive agrees
    org, dirs = po.camera_rays(spec, w, h, px)
    r = orc.trace(org, dirs)
    gtr = sc.intersection(org.astype(np.float32), dirs.astype(np.float32))
    r_gid = parity.oracle_global_prim(spec, r["obj"], r["prim"])
    g_gid = np.where(gtr["prim"] != 0xffffffff, gtr["prim"].astype(np.int64), -1)
    same = g_gid == r_gid
    print("[terrain1m lattice] primitive agrees on %.6f of %d pixels" % (same.mean(), same.size))
    assert same.mean() >= 0.9999
    od, _ = orc.render(po.DEPTH, w, h, spp=1, pixels=px)
    gd = frames[xtgpu.NODES_FP32, xtgpu.DEPTH][px[:, 1], px[:, 0]].astype(np.float64)
    hit = same & (od[:, 0] != 0)
    assert np.array_equal(gd[same & ~hit], od[same & ~hit])
    dl = np.abs(1.0 / gd[hit, 0] - 1.0 / od[hit, 0].astype(np.float64))
    print("[terrain1m depth] max |ln t_gpu - ln t_oracle| %.3g over %d pixels" % (dl.max(), hit.sum()))
    assert dl.max() <= 1e-5, np.sort(dl)[-5:]
    os_, _ = orc.render(po.STENCIL, w, h, spp=1, pixels=px)
    gs = frames[xtgpu.NODES_FP32, xtgpu.STENCIL][px[:, 1], px[:, 0]]
    assert np.array_equal(gs[same], os_[same])
    sc.close()


def test_config_hairball_2m_ao_same_stream_as_oracle():
    """Same random stream on both sides, so rays differ only where FP32 and
    FP64 part ways: AO origins leave the surface by a few hundred ulps on the
    GPU (Waechter-Binder) and by n*1e-8 in the reference, and in a hairball of
    crossing triangles a hit within that distance, or on an edge, changes."""
    spec = scenes.hairball_scene(2_000_000, seed=3)
    w = h = 1024
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8))
    img, rays = sc.render(xtgpu.AO, w, h, spp=64, ao_max_distance=0.2, seed=31)
    img2, _ = sc.render(xtgpu.AO, w, h, spp=64, ao_max_distance=0.2, seed=35)
    img8, rays8 = sc.render(xtgpu.AO, w, h, spp=64, ao_max_distance=0.2, seed=31, node_format=xtgpu.NODES_Q8)
    imgw, raysw = sc.render(xtgpu.AO, w, h, spp=64, ao_max_distance=0.2, seed=31, node_format=xtgpu.NODES_W8)
    assert np.array_equal(img, imgw) and rays == raysw
    one, _ = sc.render(xtgpu.AO, w, h, spp=1, ao_max_distance=0.2, seed=31)
    sc.close()
    assert np.all(img == img8, axis=2).mean() >= 0.9999
    assert rays == rays8
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    # per ray: one AO ray per pixel on a dense lattice, same stream
    px1 = lattice(w, h, 4)
    o1, _ = orc.render(po.AO, w, h, spp=1, ao_max_distance=0.2, seed=31, pixels=px1)
    o1b, _ = orc.render(po.AO, w, h, spp=1, ao_max_distance=0.2, seed=32, pixels=px1)
    parity.same_stream_bar(one[px1[:, 1], px1[:, 0]], o1, o1b, "hairball2m ao 1spp")
    # per pixel at 64 spp on a 32x32 lattice: same stream, and the north
    # star's bar against the 4096-spp render
    T = _truth("hairball2m_ao")
    px = T["xy"]
    o, _ = orc.render(po.AO, w, h, spp=64, ao_max_distance=0.2, seed=31, pixels=px)
    o2, _ = orc.render(po.AO, w, h, spp=64, ao_max_distance=0.2, seed=33, pixels=px)
    parity.same_stream_bar(img[px[:, 1], px[:, 0]], o, o2, "hairball2m ao 64spp")
    frames = [img[px[:, 1], px[:, 0]], img2[px[:, 1], px[:, 0]]]
    noise = T["ref_rmse"] if "ref_rmse" in T else T["oracle_rmse"]
    parity.converged_rmse_bar(np.stack(frames), T["rgba"], noise, "hairball2m ao 64spp lattice")


def test_config_precision_8m_q8_vs_fp32_vs_fp64():
    spec = scenes.precision_scene(1.0, seed=5)
    assert spec.n_tris >= 8_000_000
    w, h = 1920, 1080
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8))
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    px = lattice(w, h, 8)
    for fmt in (xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8):
        agree, rel = hits_vs_oracle(spec, sc, orc, w, h, px, fmt)
        assert agree >= 0.9999 and rel <= 1e-5, (fmt, agree, rel)
    # a 64x64 crop at 16 spp, depth 8: same stream as the oracle, and RMSE
    # against the 4096-spp render within the equal-spp noise
    T = _truth("precision_crop")
    cx = T["xy"]
    rect = (int(cx[:, 0].min()), int(cx[:, 1].min()), int(cx[:, 0].max()) + 1, int(cx[:, 1].max()) + 1)
    crops = []
    for seed in (51, 52):
        c, _ = sc.render(xtgpu.PATHTRACER, w, h, spp=16, rdepth=8, seed=seed, rect=rect, node_format=xtgpu.NODES_W8)
        crops.append(c[cx[:, 1] - rect[1], cx[:, 0] - rect[0]])
    o, _ = orc.render(po.PATHTRACER, w, h, spp=16, rdepth=8, seed=51, pixels=cx)
    o2, _ = orc.render(po.PATHTRACER, w, h, spp=16, rdepth=8, seed=53, pixels=cx)
    parity.same_stream_bar(crops[0], o, o2, "precision8m crop pt")
    parity.converged_rmse_bar(np.stack(crops), T["rgba"], T["oracle_rmse"], "precision8m crop 16spp depth 8")
    del orc
    a, ra = sc.render(xtgpu.PATHTRACER, w, h, spp=256, rdepth=8, seed=5, node_format=xtgpu.NODES_FP32)
    b, rb = sc.render(xtgpu.PATHTRACER, w, h, spp=256, rdepth=8, seed=5, node_format=xtgpu.NODES_Q8)
    c, rc = sc.render(xtgpu.PATHTRACER, w, h, spp=256, rdepth=8, seed=5, node_format=xtgpu.NODES_W8)
    assert np.array_equal(a, c) and ra == rc
    # the frame is 127 waves of 4 Mi paths; a tile of it rendered in one wave
    # gives the same pixels
    tile, _ = sc.render(xtgpu.PATHTRACER, w, h, spp=256, rdepth=8, seed=5, rect=(960, 512, 1024, 576))
    sc.close()
    assert np.array_equal(tile, a[512:576, 960:1024])
    same = np.all(a == b, axis=2)
    assert same.mean() >= 0.9999, same.mean()
    assert abs(ra - rb) <= 1e-5 * ra
