"""Converged renders (4096 samples per pixel) for the stochastic parity bars.

The pathtracer and AO integrators are judged by per-pixel RMSE against a
4096-spp render, which must sit within the sampling noise of the reference CPU
renderer at equal spp.  The reference's own equal-spp frames are in the other
fixtures (render_*.npz, made by make_golden.py from XTracer's code).  This
script makes the 4096-spp frames with the oracle (oracle/xtoracle.c, the FP64
restatement of the reference pinned to it by those fixtures): each case is
rendered as independent seeds on worker processes and the frames averaged.

It also renders, with the reference itself, the equal-spp frames of the two
full-size cases whose reference frames are not in the other fixtures:

* config1: 64 spheres and a plane, 256x256, pathtracer at 16 spp, depth 4 (the
  reference's per-seed RMSE against the truth and frame means are stored);
* hairball2m_ao: the 2M-triangle hairball, AO at distance 0.2, 64 spp, on a
  32x32 lattice of its 1024x1024 frame (two reference seeds, about 8 minutes
  each on 8 threads: the octree puts many triangles in every leaf).

For the 64x64 crop of the 8M-triangle precision scene the reference is out of
reach (its octree build of 8M triangles); the oracle's own equal-spp frames
give the noise there.

Writes tests/golden/truth.npz.  Run here:
    python tests/golden/make_truth.py [--jobs 8] [--only name,...]
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

TOTAL_SPP = 4096


def lattice(w, h, step):
    ys, xs = np.mgrid[step // 2:h:step, step // 2:w:step]
    return np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)


def cases():
    """name -> (scene factory name and args, integrator, width, height, pixels
    or None (whole frame, row-major), rdepth, ao distance, spp per worker
    task).  Pixels of the small cases are those of their golden fixture."""
    from xtracer_b200 import scenes  # noqa: F401
    g = lambda n: np.load(os.path.join(HERE, n))
    out = {}
    for name, (w, h) in (("spheres64", (64, 64)), ("terrain20k", (96, 54)), ("hairball20k", (64, 64))):
        r = g("render_%s.npz" % name)
        for md in (100.0, 0.2):
            key = "ao%g" % md
            out["%s_%s" % (name, key)] = (("small", name), "ao", w, h, r[key + "_xy"], 4, md, 256)
        if name == "spheres64":
            out["spheres64_pt"] = (("small", name), "pt", w, h, r["pt_xy"], 4, 100.0, 256)
    out["phong_pt"] = (("phong",), "pt", 65, 49, g("render_phong.npz")["pt_xy"], 4, 100.0, 256)
    out["mtl_pt"] = (("mtl",), "pt", 64, 48, g("render_mtl.npz")["pt_xy"], 4, 100.0, 256)
    t = g("render_textures.npz")
    for env in ("erp", "cubemap"):
        out["textures_%s_pt" % env] = (("textures", env), "pt", 64, 48, t["%s_pt_xy" % env], 4, 100.0, 256)
    out["dof_depth"] = (("dof",), "depth", 48, 48, g("render_cameras.npz")["dof_depth_xy"], 1, 100.0, 256)
    out["config1"] = (("config1",), "pt", 256, 256, None, 4, 100.0, 128)
    out["hairball2m_ao"] = (("hairball2m",), "ao", 1024, 1024, lattice(1024, 1024, 32), 4, 0.2, 512)
    # the 8M-triangle Phong / Blinn-Phong scene: a 64x64 crop, depth 8
    ys, xs = np.mgrid[512:576, 960:1024]
    out["precision_crop"] = (("precision",), "pt", 1920, 1080, np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32),
                             8, 100.0, 256)
    return out


def make_scene(key):
    from xtracer_b200 import scenes
    if key[0] == "small":
        return {"spheres64": lambda: scenes.spheres_scene(64, seed=1, name="spheres64"),
                "terrain20k": lambda: scenes.terrain_scene(20_000, seed=2, name="terrain20k"),
                "hairball20k": lambda: scenes.hairball_scene(20_000, seed=3, name="hairball20k")}[key[1]]()
    if key[0] == "phong":
        return scenes.phong_scene()
    if key[0] == "mtl":
        return scenes.mtl_scene()
    if key[0] == "textures":
        return scenes.textured_scene(key[1])
    if key[0] == "dof":
        cam = scenes.Camera((0.0, 3.0, -12.0), (0.0, 1.5, 0.0), (0.0, 1.0, 0.0), 50.0, flength=11.0, aperture=0.75)
        return scenes.spheres_scene(64, seed=1, name="cam_dof", camera=cam)
    if key[0] == "config1":
        return scenes.spheres_scene(64, seed=1)
    if key[0] == "hairball2m":
        return scenes.hairball_scene(2_000_000, seed=3)
    if key[0] == "precision":
        return scenes.precision_scene(1.0, seed=5)
    raise KeyError(key)


_SCENE = {}


def _work(args):
    """One worker task: `spp` samples per pixel at seed `seed`; returns the
    frame's sum over its samples (float64) and the rays traced."""
    skey, integ, w, h, px, rdepth, md, spp, seed = args
    from oracle import pyoracle as po
    if skey not in _SCENE:
        _SCENE.clear()
        _SCENE[skey] = po.OracleScene(make_scene(skey), po.XO_ACCEL_BVH)
    code = {"ao": po.AO, "pt": po.PATHTRACER, "depth": po.DEPTH}[integ]
    out, rays = _SCENE[skey].render(code, w, h, spp=spp, rdepth=rdepth, ao_max_distance=md, seed=seed, pixels=px)
    return out.astype(np.float64) * spp, rays


def truth(pool, name, case):
    skey, integ, w, h, px, rdepth, md, per = case
    if px is None:
        ys, xs = np.mgrid[0:h, 0:w]
        px = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)
    n = TOTAL_SPP // per
    # seeds of their own, far from the seeds the tests render with
    tasks = [(skey, integ, w, h, px, rdepth, md, per, 900_001 + 7919 * k) for k in range(n)]
    acc = np.zeros((px.shape[0], 4))
    rays = 0
    for frame, r in pool.imap_unordered(_work, tasks):
        acc += frame
        rays += r
    return px, (acc / TOTAL_SPP).astype(np.float32), rays


def rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64)[:, :3] - np.asarray(b, np.float64)[:, :3]) ** 2)))


def main():
    jobs = 8
    if "--jobs" in sys.argv:
        jobs = int(sys.argv[sys.argv.index("--jobs") + 1])
    only = None
    if "--only" in sys.argv:
        only = set(sys.argv[sys.argv.index("--only") + 1].split(","))
    path = os.path.join(HERE, "truth.npz")
    out = dict(np.load(path)) if os.path.exists(path) else {}
    from oracle import pyoracle as po
    ctx = mp.get_context("spawn")
    with ctx.Pool(jobs) as pool:
        for name, case in cases().items():
            if only and name not in only:
                continue
            t0 = time.time()
            px, img, rays = truth(pool, name, case)
            out[name + "_xy"], out[name + "_rgba"] = px, img
            out[name + "_spp"] = np.int64(TOTAL_SPP)
            print(name, "%.1fs" % (time.time() - t0), rays, "rays", flush=True)
            if name == "config1":
                # the reference at equal spp (16, depth 4) on the whole frame
                spec = make_scene(case[0])
                work = tempfile.mkdtemp(prefix="xttruth")
                scn = spec.write_scn(work)
                by = {tuple(p): i for i, p in enumerate(px.tolist())}
                rm, means = [], []
                for seed in (61, 62, 63, 64):
                    xy, rgba, st = po.ref_render(scn, "pathtracer", 256, 256, spp=16, rdepth=4, threads=jobs,
                                                 seed=seed, workdir=work)
                    order = np.array([by[tuple(p)] for p in xy.tolist()])
                    rm.append(rmse(rgba, img[order]))
                    means.append(rgba[:, :3].astype(np.float64).mean(0))
                out["config1_ref_rmse"] = np.array(rm)
                out["config1_ref_mean"] = np.array(means)
                out["config1_ref_spp"] = np.int64(16)
                print("config1 reference RMSE at 16 spp", rm, flush=True)
            if name == "hairball2m_ao":
                spec = make_scene(case[0])
                work = tempfile.mkdtemp(prefix="xttruth")
                scn = spec.write_scn(work)
                by = {tuple(p): i for i, p in enumerate(px.tolist())}
                tiles = [(x, y, x + 1, y + 1) for x, y in px.tolist()]
                rm, means = [], []
                for seed in (65, 66):
                    t1 = time.time()
                    xy, rgba, st = po.ref_render(scn, "ao", 1024, 1024, spp=64, threads=jobs, seed=seed, tiles=tiles,
                                                 ao_max_distance=0.2, workdir=work)
                    order = np.array([by[tuple(p)] for p in xy.tolist()])
                    rm.append(rmse(rgba, img[order]))
                    means.append(rgba[:, :3].astype(np.float64).mean(0))
                    print("hairball2m_ao reference seed", seed, "%.0fs" % (time.time() - t1), st, flush=True)
                out["hairball2m_ao_ref_rmse"] = np.array(rm)
                out["hairball2m_ao_ref_mean"] = np.array(means)
                out["hairball2m_ao_ref_spp"] = np.int64(64)
                print("hairball2m_ao reference RMSE at 64 spp", rm, flush=True)
            if name in ("hairball2m_ao", "precision_crop"):
                # equal-spp noise from the oracle at seeds of its own
                spp = 64 if name == "hairball2m_ao" else 16
                skey, integ, w, h, _, rdepth, md, _ = case
                tasks = [(skey, integ, w, h, px, rdepth, md, spp, 700_001 + 31 * k) for k in range(4)]
                frames = [f / spp for f, _ in pool.imap(_work, tasks)]
                out[name + "_oracle_rmse"] = np.array([rmse(f, img) for f in frames])
                out[name + "_oracle_mean"] = np.array([f[:, :3].mean(0) for f in frames])
                out[name + "_oracle_spp"] = np.int64(spp)
                print(name, "oracle RMSE at %d spp" % spp, out[name + "_oracle_rmse"], flush=True)
    tmp = os.path.join(HERE, "truth.partial.npz")
    np.savez_compressed(tmp, **out)
    os.replace(tmp, path)
    print("truth.npz", sorted(out))


if __name__ == "__main__":
    main()
