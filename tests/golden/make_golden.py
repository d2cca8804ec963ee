"""Generates the golden fixtures in tests/golden/ by running the REFERENCE
renderer's own code (XTracer's xtcore compiled from its sources by
oracle/ref.mk, driven by oracle/ref_driver.cc).

The reference ships no unit tests, golden images or known-answer vectors, so
these fixtures are what pins the oracle restatement (oracle/xtoracle.c):

* kat.npz     single reference functions on seeded and edge-case inputs
              (camera, sphere, plane, triangle, AABB, hemisphere, diffuse, lobe,
              Lambert/Phong/Blinn-Phong/Emissive sample_path, gradient sky),
              with the libc rand() values each sampling call consumed;
* hits_*.npz  primary-ray closest hits (object, triangle index from an
              Octree<Triangle> replica, t, point, normal) on small scenes;
* render_*.npz stencil/depth frames (deterministic) and AO/pathtracer frames at
              several seeds (single thread, time() fixed by the driver) for the
              statistical checks;
* render_primary_*.npz  frames of the normal, uv, emission and wireframe
              integrators (deterministic, 3 samples per pixel) on scenes that
              exercise every texture-coordinate path (`--primary` regenerates
              only these);
* kat_cameras.npz, render_cameras.npz  rays of the ERP, ODS, cubemap and
              depth-of-field cameras (with the rand() values the latter drew),
              and stencil/depth/normal frames through each camera with grid
              anti-aliasing (`--cameras` regenerates only these);
* kat_textures.npz, render_textures.npz  Texture2D (nearest and bilinear,
              flipped), ERP and Cubemap samples on PNG files the reference
              loads, and frames of textured scenes with ERP and cubemap
              environments: emission and depth-1 pathtracer (deterministic)
              and depth-4 pathtracer at four seeds (`--textures`);
* raygraph.npz  the depth integrator's raygraph exported as PLY the way the GUI
              does it (render::assemble + raygraph::write), with the frame
              (`--raygraph`);
* render_mtl.npz  frames of meshes loaded from an OBJ with an MTL library
              (BlinnPhong / Emissive materials, map_Kd / map_Ks / map_Ke
              textures): depth, uv, emission, depth-1 pathtracer, and a
              depth-4 pathtracer at four seeds (`--mtl`);
* render_random.npz  stencil and depth frames with the random sample
              distribution (aa.cc:34-48) at four seeds, one reproducible set of
              rand() jitter offsets each (`--random`);
* render_phong.npz  depth-4 pathtracer frames of Phong and Blinn-Phong
              spheres and plane (reflectance 0.5 and 1, exponents 8 and 256)
              at four seeds, and known answers of sample::lobe where its frame
              is the identity (direction along the normal) or its result
              underflows (`--phong`).

Run here (needs the reference sources and oracle/_ref/xtref):
    make -f oracle/ref.mk REF=<xtracer source tree> -j8
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from xtracer_b200 import scenes  # noqa: E402

H = float.hex


def _line(kind, *vals):
    return " ".join([kind] + [H(float(v)) for v in vals])


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def make_kat(rng):
    out = {}
    # --- camera (perspective.cc:38-98)
    cam_in = []
    for i in range(64):
        pos = rng.uniform(-20, 20, 3).astype(np.float32)
        tgt = (pos + rng.uniform(-10, 10, 3)).astype(np.float32)
        up = np.array([0, 1, 0], np.float32) if i % 4 else rng.uniform(-1, 1, 3).astype(np.float32)
        fov = np.float32(rng.choice([30.0, 45.0, 60.0, 90.0, 37.5]))
        w, h = [(256, 256), (1920, 1080), (64, 48), (1024, 1024)][i % 4]
        x, y = np.float32(rng.integers(0, w) + 0.5), np.float32(rng.integers(0, h) + 0.5)
        cam_in.append(np.concatenate([pos, tgt, up, [fov, w, h, x, y]]).astype(np.float64))
    cam_in = np.array(cam_in)
    res = po.ref_kat([_line("camera", *r) for r in cam_in])
    out["camera_in"] = cam_in
    out["camera_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])

    # --- sphere (sphere.cc:35-62)
    sph = []
    for i in range(200):
        c = rng.uniform(-5, 5, 3); r = rng.uniform(0.1, 2.0)
        if i % 5 == 0:
            o = c + _unit(rng, 1)[0] * r * 0.5            # origin inside -> miss
        else:
            o = c + _unit(rng, 1)[0] * rng.uniform(r * 1.5, 10)
        if i % 3 == 0:
            d = c + _unit(rng, 1)[0] * r * 0.7 - o          # towards the sphere
        else:
            d = _unit(rng, 1)[0]
        d = d / np.linalg.norm(d)
        sph.append(np.concatenate([c, [r], o, d]))
    sph += [np.array([0, 0, 0, 1, -5, 1, 0, 1, 0, 0.0]),   # tangent: discriminant 0
            np.array([0, 0, 0, 0, -5, 0, 0, 1, 0, 0.0]),   # radius 0 (point light)
            np.array([0, 0, 5, 1, 0, 0, 0, 0, 0, 1.0]),    # axis ray
            np.array([0, 0, -5, 1, 0, 0, 0, 0, 0, 1.0])]   # sphere behind
    sph = np.array(sph)
    res = po.ref_kat([_line("sphere", *r) for r in sph])
    out["sphere_in"] = sph
    out["sphere_out"] = np.array([[int(r[1])] + [float.fromhex(t) for t in r[2:]] for r in res])

    # --- plane (plane.cc:19-61)
    pl = []
    for i in range(100):
        n = _unit(rng, 1)[0] if i % 4 else np.array([0, 1, 0.0])
        off = rng.uniform(-3, 3)
        o = rng.uniform(-5, 5, 3)
        d = _unit(rng, 1)[0]
        pl.append(np.concatenate([n, [off], o, d]))
    pl += [np.array([0, 1, 0, 0, 0, 1, 0, 1, 0, 0.0]),     # parallel
           np.array([0, 1, 0, 0, 0, -1, 0, 0, 1, 0.0]),    # from below (two-sided)
           np.array([0, 1, 0, 2, 0, 5, 0, 0, -1, 0.0])]    # offset plane
    pl = np.array(pl)
    res = po.ref_kat([_line("plane", *r) for r in pl])
    out["plane_in"] = pl
    out["plane_out"] = np.array([[int(r[1])] + [float.fromhex(t) for t in r[2:]] for r in res])

    # --- triangle (triangle.cc:82-184)
    tri = []
    for i in range(300):
        v = rng.uniform(-3, 3, (3, 3))
        nrm = np.zeros((3, 3)) if i % 3 else _unit(rng, 3)
        bc = rng.dirichlet([1, 1, 1])
        if i % 7 == 0:
            bc = np.array([0.5, 0.5, 0.0])                  # on an edge
        if i % 11 == 0:
            bc = np.array([1.0, 0.0, 0.0])                  # on a vertex
        if i % 13 == 0:
            bc = np.array([1.2, -0.1, -0.1])                # outside
        p = bc @ v
        o = p + _unit(rng, 1)[0] * rng.uniform(0.5, 8)
        d = (p - o) / np.linalg.norm(p - o)
        if i % 17 == 0:
            d = -d                                          # pointing away
        tri.append(np.concatenate([v.ravel(), nrm.ravel(), o, d]))
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0.0]])
    tri += [np.concatenate([v.ravel(), np.zeros(9), [0.2, 0.2, -1], [1, 0, 0]]),      # parallel
            np.concatenate([np.zeros(9), np.zeros(9), [0, 0, -1], [0, 0, 1]])]          # degenerate
    tri = np.array(tri)
    res = po.ref_kat([_line("triangle", *r) for r in tri])
    out["triangle_in"] = tri
    out["triangle_out"] = np.array([[int(r[1])] + [float.fromhex(t) for t in r[2:]] for r in res])

    # --- AABB slab test (aabb.cc:32-71)
    bb = []
    for i in range(300):
        a = rng.uniform(-3, 3, 3); b = a + rng.uniform(0.01, 3, 3)
        o = rng.uniform(-6, 6, 3)
        d = _unit(rng, 1)[0]
        if i % 5 == 0:
            d[rng.integers(0, 3)] = 0.0
            d /= np.linalg.norm(d)
        if i % 9 == 0:
            o = (a + b) / 2                                 # inside
        bb.append(np.concatenate([a, b, o, d]))
    bb = np.array(bb)
    res = po.ref_kat([_line("aabb", *r) for r in bb])
    out["aabb_in"] = bb
    out["aabb_out"] = np.array([int(r[1]) for r in res])

    # --- sampling with the rand() values they consume
    seeds = np.arange(1, 97, dtype=np.int64) * 7919
    res = po.ref_kat(["rand %d 64" % s for s in seeds])
    out["rand_seeds"] = seeds
    out["rand_table"] = np.array([[int(t) for t in r[1:65]] for r in res], np.int64)
    out["rand_max"] = np.int64(int(res[0][65]))
    nrm = _unit(rng, 96)
    nrm[0] = [0, 1, 0]; nrm[1] = [0, 0, 1]; nrm[2] = [1, 0, 0]
    res = po.ref_kat(["hemisphere %d %s %s %s" % (s, H(n[0]), H(n[1]), H(n[2])) for s, n in zip(seeds, nrm)])
    out["hemisphere_n"] = nrm
    out["hemisphere_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    res = po.ref_kat(["diffuse %d %s %s %s" % (s, H(n[0]), H(n[1]), H(n[2])) for s, n in zip(seeds, nrm)])
    out["diffuse_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    dirs = _unit(rng, 96)
    dirs = np.where((np.sum(dirs * nrm, axis=1) < 0)[:, None], -dirs, dirs)
    exps = rng.uniform(1, 256, 96)
    res = po.ref_kat(["lobe %d %s %s %s %s %s %s %s" % ((s,) + tuple(H(x) for x in n) + tuple(H(x) for x in d) + (H(e),))
                      for s, n, d, e in zip(seeds, nrm, dirs, exps)])
    out["lobe_d"] = dirs
    out["lobe_e"] = exps
    out["lobe_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])

    # --- materials (lambert.cc:30-40, phong.cc:35-55, blinnphong.cc:34-61, emissive.cc:20-27)
    mat_in = []
    for i, s in enumerate(seeds):
        mtype = i % 4
        cols = rng.uniform(0, 1, 9).astype(np.float32)
        refl = np.float32(rng.choice([0.0, 0.25, 0.5, 0.75, 1.0]))
        ex = np.float32(rng.uniform(8, 256))
        p = rng.uniform(-5, 5, 3)
        n = nrm[i]
        inc = -dirs[i]
        mat_in.append(np.concatenate([[mtype, s], cols, [refl, ex], p, n, inc]))
    mat_in = np.array(mat_in)
    res = po.ref_kat([" ".join(["material", str(int(r[0])), str(int(r[1]))] + [H(float(x)) for x in r[2:]])
                      for r in mat_in])
    out["material_in"] = mat_in
    out["material_out"] = np.array([[int(r[1])] + [float.fromhex(t) for t in r[2:]] for r in res])

    # --- gradient environment (sampler_gradient.cc:11-17)
    g_in = np.concatenate([rng.uniform(0, 1, (64, 6)).astype(np.float32).astype(np.float64), _unit(rng, 64)], axis=1)
    res = po.ref_kat([_line("gradient", *r) for r in g_in])
    out["gradient_in"] = g_in
    out["gradient_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    return out


def small_scenes():
    """Small scenes for the fixtures (names double as fixture names)."""
    sp = scenes.spheres_scene(64, seed=1, name="spheres64")
    te = scenes.terrain_scene(20_000, seed=2, name="terrain20k")
    hb = scenes.hairball_scene(20_000, seed=3, name="hairball20k")
    return {"spheres64": (sp, 64, 64), "terrain20k": (te, 96, 54), "hairball20k": (hb, 64, 64)}


def primary_scenes():
    return {"spheres64": (scenes.spheres_scene(64, seed=1, name="spheres64"), 64, 64),
            "terrain20k": (scenes.terrain_scene(20_000, seed=2, name="terrain20k"), 96, 54),
            "uvscene": (scenes.uv_scene(6), 80, 60)}


def make_primary(work):
    for name, (spec, w, h) in primary_scenes().items():
        scn = spec.write_scn(work)
        rend = {}
        for integ in ("normal", "uv", "emission", "wireframe"):
            xy, rgba, st = po.ref_render(scn, integ, w, h, spp=3, threads=1, seed=1, workdir=work)
            rend["%s_xy" % integ] = xy
            rend["%s_rgba" % integ] = rgba
            rend["%s_rays" % integ] = st["rays"]
        np.savez_compressed(os.path.join(HERE, "render_primary_%s.npz" % name), width=w, height=h, spp=3, **rend)
        print("render_primary", name, sorted(rend))


def make_cameras(work, rng):
    kat = {}
    # equirectangular and omni-directional stereo (camera/erp.cc, ods.cc)
    for kind in ("erp", "ods"):
        rows = []
        for i in range(96):
            pos = rng.uniform(-5, 5, 3)
            ori = rng.uniform(-np.pi, np.pi, 3) if i % 4 else np.zeros(3)
            ipd = rng.uniform(0.05, 0.2)
            w, h = [(128, 64), (256, 256), (64, 48), (1000, 500)][i % 4]
            x, y = rng.uniform(0, w), rng.uniform(0, h)
            rows.append(np.concatenate([pos, ori, [ipd, w, h, x, y]]).astype(np.float32).astype(np.float64))
        rows = np.array(rows)
        res = po.ref_kat([_line("camera_" + kind, *r) for r in rows])
        kat[kind + "_in"] = rows
        kat[kind + "_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    # cubemap vertical strip (camera/cubemap.cc)
    rows = []
    for i in range(96):
        pos = rng.uniform(-5, 5, 3)
        w = [16, 64, 100, 31][i % 4]
        h = 6 * [16, 64, 100, 7][i % 4]
        x, y = rng.uniform(0, w), rng.uniform(0, h)
        rows.append(np.concatenate([pos, [w, h, x, y]]).astype(np.float32).astype(np.float64))
    rows = np.array(rows)
    res = po.ref_kat([_line("camera_cubemap", *r) for r in rows])
    kat["cubemap_in"] = rows
    kat["cubemap_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    # perspective with depth of field (perspective.cc:73-95): two prng_c draws
    rows, seeds = [], rng.integers(1, 2 ** 31 - 1, 96)
    for i in range(96):
        pos = rng.uniform(-10, 10, 3); tgt = pos + rng.uniform(-5, 5, 3)
        up = np.array([0, 1, 0.0]) if i % 3 else rng.uniform(-1, 1, 3)
        fov = rng.choice([30.0, 45.0, 60.0]); fl = rng.uniform(0.5, 20.0); ap = rng.uniform(0.0, 2.0)
        w, h = [(64, 64), (1920, 1080), (100, 50)][i % 3]
        x, y = rng.uniform(0, w), rng.uniform(0, h)
        rows.append(np.concatenate([[seeds[i]], pos, tgt, up, [fov, fl, ap, w, h, x, y]]).astype(np.float32)
                    .astype(np.float64))
    rows = np.array(rows)
    rows[:, 0] = seeds
    res = po.ref_kat([_line("camera_dof", *r) for r in rows])
    kat["dof_in"] = rows
    kat["dof_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    tab = po.ref_kat(["rand %d 8" % s for s in seeds])
    kat["dof_table"] = np.array([[int(t) for t in r[1:9]] for r in tab], np.int64)
    kat["rand_max"] = int(tab[0][9])
    np.savez_compressed(os.path.join(HERE, "kat_cameras.npz"), **kat)
    print("kat_cameras.npz", {k: np.shape(v) for k, v in kat.items()})
    # frames through each camera, grid anti-aliasing
    rend = {}
    for tag, cam, w, h, aa in camera_cases():
        spec = scenes.spheres_scene(64, seed=1, name="cam_" + tag, camera=cam)
        scn = spec.write_scn(work)
        for integ in ("stencil", "depth", "normal"):
            xy, rgba, st = po.ref_render(scn, integ, w, h, spp=2, aa=aa, threads=1, seed=1, workdir=work)
            rend["%s_%s_xy" % (tag, integ)] = xy
            rend["%s_%s_rgba" % (tag, integ)] = rgba
            rend["%s_%s_rays" % (tag, integ)] = st["rays"]
    dof = scenes.Camera((0.0, 3.0, -12.0), (0.0, 1.5, 0.0), (0.0, 1.0, 0.0), 50.0, flength=11.0, aperture=0.75)
    spec = scenes.spheres_scene(64, seed=1, name="cam_dof", camera=dof)
    scn = spec.write_scn(work)
    imgs = []
    for seed in (31, 32, 33, 34):
        xy, rgba, st = po.ref_render(scn, "depth", 48, 48, spp=16, threads=1, seed=seed, workdir=work)
        imgs.append(rgba)
    rend["dof_depth_xy"] = xy
    rend["dof_depth_rgba"] = np.stack(imgs)
    np.savez_compressed(os.path.join(HERE, "render_cameras.npz"), **rend)
    print("render_cameras.npz", sorted(rend))


def sampler_kat_textures(rng):
    """The textures of the sampler known-answer vectors: (pixels, filtering,
    flip_x, flip_y) with odd sizes, RGB and RGBA, both filters and flips."""
    out = []
    for i, (h, w, c) in enumerate([(5, 7, 3), (6, 9, 4), (8, 8, 3), (1, 3, 3), (4, 16, 4), (3, 1, 3)]):
        out.append((rng.integers(0, 256, (h, w, c), dtype=np.uint8), i % 2, int(i in (1, 4)), int(i in (2, 4))))
    return out


def make_textures(work, rng):
    """Sampler known-answer vectors (Texture2D nearest / bilinear, ERP,
    Cubemap on PNG files loaded by the reference) and frames of the textured
    scenes rendered by the reference."""
    kat = {}
    texs = sampler_kat_textures(rng)
    lines = []
    for i, (px, filt, fx, fy) in enumerate(texs):
        path = os.path.join(work, "kat_t%d.png" % i)
        scenes.write_png(path, px)
        lines.append("tex_load %d %d %d %d %s" % (i, filt, fx, fy, path))
        kat["tex%d_pixels" % i] = px
        kat["tex%d_mode" % i] = np.array([filt, fx, fy], np.int32)
    uv = np.concatenate([rng.uniform(-2.5, 2.5, (160, 2)), rng.uniform(0, 1, (160, 2)),
                         np.array([[0, 0], [1, 1], [0.5, 1], [1, 0.5], [-0.0, 0.25], [2, -1], [3.75, -2.25],
                                   [np.nan, 0.5], [0.5, np.nan], [np.inf, 0.5], [-np.inf, 0.5], [1e10, -1e10]])])
    rows = []
    for i in range(len(texs)):
        for u, v in uv:
            lines.append("tex_sample %d %s %s" % (i, H(float(u)), H(float(v))))
            rows.append((i, u, v))
    erp = rng.integers(0, 256, (9, 17, 3), dtype=np.uint8)
    faces = [rng.integers(0, 256, (4 + k % 3, 5 + k % 2, 3), dtype=np.uint8) for k in range(6)]
    scenes.write_png(os.path.join(work, "kat_erp.png"), erp)
    fpaths = []
    for k, f in enumerate(faces):
        fpaths.append(os.path.join(work, "kat_face%d.png" % k))
        scenes.write_png(fpaths[-1], f)
    lines += ["erp_load 0 %s" % os.path.join(work, "kat_erp.png"), "cube_load 0 %s" % " ".join(fpaths)]
    dirs = np.concatenate([rng.normal(size=(300, 3)),
                           np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                                     [0, 0, 0], [1, 1, 0], [1, -1, 1], [0.5, 0.5, -0.5], [np.nan, 0, 1]])])
    for v in dirs:
        lines.append(_line("erp_sample", 0, *v))
        lines.append(_line("cube_sample", 0, *v))
    res = po.ref_kat(lines)
    assert all(r[1:] == ["0"] for r in res if r[0] in ("tex_load", "erp_load")), "texture load failed"
    tex_out = [[float.fromhex(t) for t in r[1:4]] for r in res if r[0] == "tex_sample"]
    kat["tex_in"] = np.array(rows, np.float64)
    kat["tex_out"] = np.array(tex_out, np.float32)
    kat["erp_pixels"] = erp
    for k, f in enumerate(faces):
        kat["face%d_pixels" % k] = f
    kat["dirs"] = dirs
    kat["erp_out"] = np.array([[float.fromhex(t) for t in r[1:4]] for r in res if r[0] == "erp_sample"], np.float32)
    kat["cube_out"] = np.array([[float.fromhex(t) for t in r[1:4]] for r in res if r[0] == "cube_sample"], np.float32)
    np.savez_compressed(os.path.join(HERE, "kat_textures.npz"), **kat)
    print("kat_textures.npz", sorted(kat))

    rend = {}
    for env in ("erp", "cubemap"):
        spec = scenes.textured_scene(env)
        scn = spec.write_scn(work)
        w, h = texture_frame_size()
        # emission folds each sample's emissive texel; a pathtracer of depth 1
        # returns the environment's texel on a miss and the emissive sampler's
        # on an emissive hit (eval(0) is black), so both are deterministic
        for integ, spp, rdepth, aa in (("emission", 2, 1, 2), ("pathtracer", 2, 1, 1)):
            xy, rgba, st = po.ref_render(scn, integ, w, h, spp=spp, rdepth=rdepth, aa=aa, threads=1, seed=1,
                                         workdir=work)
            rend["%s_%s_xy" % (env, integ)] = xy
            rend["%s_%s_rgba" % (env, integ)] = rgba
            rend["%s_%s_rays" % (env, integ)] = st["rays"]
        imgs = []
        for seed in (51, 52, 53, 54):
            xy, rgba, st = po.ref_render(scn, "pathtracer", w, h, spp=16, rdepth=4, threads=1, seed=seed,
                                         workdir=work)
            imgs.append(rgba)
        rend["%s_pt_xy" % env] = xy
        rend["%s_pt_rgba" % env] = np.stack(imgs)
    np.savez_compressed(os.path.join(HERE, "render_textures.npz"), **rend)
    print("render_textures.npz", sorted(rend))


def raygraph_case():
    """(scene, width, height, spp, aa) of the raygraph fixture: partial tiles,
    grid anti-aliasing, hits and misses."""
    return scenes.spheres_scene(16, seed=1, name="raygraph"), 40, 24, 1, 2


def make_raygraph(work):
    """The depth integrator's raygraph as the GUI exports it (assemble +
    raygraph::write) from the reference's own render."""
    spec, w, h, spp, aa = raygraph_case()
    scn = spec.write_scn(work)
    ply = os.path.join(work, "raygraph.ply")
    xy, rgba, st = po.ref_render(scn, "depth", w, h, spp=spp, aa=aa, threads=1, workdir=work, raygraph=ply)
    text = open(ply, "rb").read()
    np.savez_compressed(os.path.join(HERE, "raygraph.npz"), ply=np.frombuffer(text, np.uint8), xy=xy, rgba=rgba)
    print("raygraph.npz", len(text), "bytes of PLY")


def make_mtl(work):
    """Frames of the OBJ-with-MTL scene (meshes through the loader's external
    object path): deterministic depth, uv, emission and depth-1 pathtracer,
    and a depth-4 pathtracer at four seeds."""
    spec = scenes.mtl_scene()
    scn = spec.write_scn(work)
    rend = {}
    for integ, rdepth in (("depth", 1), ("uv", 1), ("emission", 1), ("pathtracer", 1)):
        xy, rgba, st = po.ref_render(scn, integ, 64, 48, spp=2, rdepth=rdepth, threads=1, workdir=work)
        rend["%s_xy" % integ], rend["%s_rgba" % integ], rend["%s_rays" % integ] = xy, rgba, st["rays"]
    imgs = []
    for seed in (71, 72, 73, 74):
        xy, rgba, st = po.ref_render(scn, "pathtracer", 64, 48, spp=16, rdepth=4, threads=1, seed=seed,
                                     workdir=work)
        imgs.append(rgba)
    rend["pt_xy"], rend["pt_rgba"] = xy, np.stack(imgs)
    np.savez_compressed(os.path.join(HERE, "render_mtl.npz"), **rend)
    print("render_mtl.npz", sorted(rend))


def random_case():
    """(camera, width, height, spp, (integrator, aa) pairs, seeds) of the random
    sample distribution fixture."""
    cam = scenes.Camera((0.0, 6.0, -14.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 60.0)
    return cam, 48, 40, 2, [("stencil", 1), ("stencil", 4), ("depth", 4)], (41, 42, 43, 44)


def make_random(work):
    """Frames of the random sample distribution (aa.cc:34-48): the reference
    seeds rand() from time(), which the driver fixes to the given seed, so
    each seed is one reproducible draw of the jitter offsets."""
    cam, w, h, spp, cases, seeds = random_case()
    spec = scenes.spheres_scene(64, seed=1, name="cam_random", camera=cam)
    scn = spec.write_scn(work)
    rend = {}
    for integ, aa in cases:
        imgs, rays = [], []
        for seed in seeds:
            xy, rgba, st = po.ref_render(scn, integ, w, h, spp=spp, aa=aa, threads=1, seed=seed, workdir=work,
                                         distribution=po.SAMPLES_RANDOM)
            imgs.append(rgba)
            rays.append(st["rays"])
        rend["%s_aa%d_xy" % (integ, aa)] = xy
        rend["%s_aa%d_rgba" % (integ, aa)] = np.stack(imgs)
        rend["%s_aa%d_rays" % (integ, aa)] = np.array(rays, np.int64)
    np.savez_compressed(os.path.join(HERE, "render_random.npz"), **rend)
    print("render_random.npz", sorted(rend))


def phong_case():
    """(scene, width, height, spp, depth, seeds) of the Phong fixture; odd
    width and height put the centre pixel's ray on the camera axis."""
    return scenes.phong_scene(), 65, 49, 16, 4, (51, 52, 53, 54)


def lobe_edge_cases(rng):
    """(seed, normal, direction, exponent) rows for sample::lobe at the edges
    of sample.inl:61-90: the direction equal to the normal (identity frame),
    1 - d.n just below and just above 1e-8, and exponents up to 2000, where
    pow(vdotr, e) underflows."""
    rows = []
    seeds = np.arange(1, 65, dtype=np.int64) * 104729
    for i, sd in enumerate(seeds):
        n = _unit(rng, 1)[0]
        if i % 8 == 0:
            n = np.array([0.0, 0.0, -1.0])
        e = [8.0, 64.0, 256.0, 2000.0][i % 4]
        kind = (i // 4) % 4
        if kind == 0:
            d = n.copy()
        else:
            # rotate n by an angle whose 1 - cos is 5e-9, 2e-8 or 1e-3
            ang = {1: np.arccos(1 - 5e-9), 2: np.arccos(1 - 2e-8), 3: np.arccos(1 - 1e-3)}[kind]
            a = np.cross(n, _unit(rng, 1)[0])
            a /= np.linalg.norm(a)
            d = n * np.cos(ang) + np.cross(a, n) * np.sin(ang)
        rows.append((int(sd), n, d, e))
    return rows


def make_phong(work):
    """Depth-4 pathtracer frames of the Phong scene at four seeds, and
    sample::lobe known answers at its edges with the rand() values each call
    consumed."""
    spec, w, h, spp, depth, seeds = phong_case()
    scn = spec.write_scn(work)
    rend = {}
    imgs, rays = [], []
    for seed in seeds:
        xy, rgba, st = po.ref_render(scn, "pathtracer", w, h, spp=spp, rdepth=depth, threads=1, seed=seed,
                                     workdir=work)
        imgs.append(rgba)
        rays.append(st["rays"])
    rend["pt_xy"], rend["pt_rgba"], rend["pt_rays"] = xy, np.stack(imgs), np.array(rays, np.int64)
    rows = lobe_edge_cases(np.random.default_rng(20261206))
    res = po.ref_kat(["rand %d 8" % r[0] for r in rows])
    rend["lobe_rand"] = np.array([[int(t) for t in r[1:9]] for r in res], np.int64)
    rend["rand_max"] = np.int64(int(res[0][9]))
    res = po.ref_kat(["lobe %d %s %s %s %s %s %s %s" % ((r[0],) + tuple(H(float(x)) for x in r[1]) +
                                                        tuple(H(float(x)) for x in r[2]) + (H(r[3]),))
                      for r in rows])
    rend["lobe_n"] = np.array([r[1] for r in rows])
    rend["lobe_d"] = np.array([r[2] for r in rows])
    rend["lobe_e"] = np.array([r[3] for r in rows])
    rend["lobe_out"] = np.array([[float.fromhex(t) for t in r[1:]] for r in res])
    np.savez_compressed(os.path.join(HERE, "render_phong.npz"), width=w, height=h, spp=spp, depth=depth,
                        seeds=np.array(seeds), **rend)
    print("render_phong.npz", sorted(rend))


def texture_frame_size():
    return 64, 48


def camera_cases():
    """(tag, camera, width, height, aa) of the camera frame fixtures."""
    C = scenes.Camera
    return [("persp_aa3", C((0.0, 6.0, -14.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 60.0), 48, 40, 3),
            ("erp_aa2", C((0.5, 2.0, 0.25), type=scenes.CAM_ERP, orientation=(0.25, -0.5, 0.125)), 96, 48, 2),
            ("ods_aa2", C((0.5, 2.0, 0.25), type=scenes.CAM_ODS, orientation=(0.0, 0.75, 0.0), ipd=0.125),
             64, 64, 2),
            ("cubemap_aa2", C((0.5, 2.0, 0.25), type=scenes.CAM_CUBEMAP), 24, 144, 2)]


def main():
    if not po.ref_available():
        raise SystemExit("oracle/_ref/xtref missing: make -f oracle/ref.mk REF=<xtracer sources>")
    if "--primary" in sys.argv:
        make_primary(tempfile.mkdtemp(prefix="xtgold"))
        return
    if "--cameras" in sys.argv:
        make_cameras(tempfile.mkdtemp(prefix="xtgold"), np.random.default_rng(20261204))
        return
    if "--mtl" in sys.argv:
        make_mtl(tempfile.mkdtemp(prefix="xtgold"))
        return
    if "--raygraph" in sys.argv:
        make_raygraph(tempfile.mkdtemp(prefix="xtgold"))
        return
    if "--phong" in sys.argv:
        make_phong(tempfile.mkdtemp(prefix="xtgold"))
        return
    if "--random" in sys.argv:
        make_random(tempfile.mkdtemp(prefix="xtgold"))
        return
    if "--textures" in sys.argv:
        make_textures(tempfile.mkdtemp(prefix="xtgold"), np.random.default_rng(20261205))
        return
    rng = np.random.default_rng(20261203)
    kat = make_kat(rng)
    np.savez_compressed(os.path.join(HERE, "kat.npz"), **kat)
    print("kat.npz", {k: v.shape for k, v in kat.items()})
    if "--kat-only" in sys.argv:
        return

    work = tempfile.mkdtemp(prefix="xtgold")
    for name, (spec, w, h) in small_scenes().items():
        scn = spec.write_scn(work)
        objp = spec.mesh_obj_path(work, 0) if spec.n_tris else None
        hits = po.ref_hits(scn, w, h, None, objp, workdir=work)
        names = np.array(hits.pop("names"))
        np.savez_compressed(os.path.join(HERE, "hits_%s.npz" % name), names=names, width=w, height=h, **hits)
        print("hits", name, int(hits["hit"].sum()), "hits of", hits["hit"].size)
        rend = {}
        for integ, spp in (("stencil", 2), ("depth", 2)):
            xy, rgba, st = po.ref_render(scn, integ, w, h, spp=spp, threads=1, seed=1, workdir=work)
            rend["%s_xy" % integ] = xy
            rend["%s_rgba" % integ] = rgba
            rend["%s_spp" % integ] = spp
        # AO: the shipped distance (100) and the hairball workload's 0.2;
        # four seeds each so the reference's own noise can be estimated.
        for md in (100.0, 0.2):
            tag = "ao%g" % md
            imgs = []
            for seed in (11, 12, 13, 14):
                xy, rgba, st = po.ref_render(scn, "ao", w, h, spp=16, threads=1, seed=seed,
                                             ao_max_distance=md, workdir=work)
                imgs.append(rgba)
            rend["%s_xy" % tag] = xy
            rend["%s_rgba" % tag] = np.stack(imgs)
            rend["%s_spp" % tag] = 16
        if name == "spheres64":
            imgs = []
            for seed in (21, 22, 23, 24):
                xy, rgba, st = po.ref_render(scn, "pathtracer", w, h, spp=16, rdepth=4, threads=1, seed=seed,
                                             workdir=work)
                imgs.append(rgba)
                rend["pt_rays_seed%d" % seed] = st["rays"]
            rend["pt_xy"] = xy
            rend["pt_rgba"] = np.stack(imgs)
            rend["pt_spp"] = 16
            rend["pt_depth"] = 4
        np.savez_compressed(os.path.join(HERE, "render_%s.npz" % name), width=w, height=h, **rend)
        print("render", name, sorted(rend))


if __name__ == "__main__":
    main()
