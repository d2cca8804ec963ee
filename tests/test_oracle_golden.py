"""Pins the oracle restatement (oracle/xtoracle.c) against fixtures made by the
reference renderer's own code (tests/golden/make_golden.py).

Deterministic functions must match bit for bit; AO and pathtracer frames use a
different random source than the reference's libc rand(), so they must agree
within the reference's own sampling noise at equal spp.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from xtracer_b200 import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def P(a):
    return np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def kat():
    return np.load(os.path.join(GOLD, "kat.npz"))


def small_scenes():
    return {"spheres64": (scenes.spheres_scene(64, seed=1, name="spheres64"), 64, 64),
            "terrain20k": (scenes.terrain_scene(20_000, seed=2, name="terrain20k"), 96, 54),
            "hairball20k": (scenes.hairball_scene(20_000, seed=3, name="hairball20k"), 64, 64)}


def test_camera_kat(kat):
    L = po.lib()
    for r, o in zip(kat["camera_in"], kat["camera_out"]):
        pos, tgt, up = [(C.c_float * 3)(*r[i:i + 3]) for i in (0, 3, 6)]
        org = np.zeros(3); d = np.zeros(3)
        L.xo_camera_ray(C.cast(pos, C.c_void_p), C.cast(tgt, C.c_void_p), C.cast(up, C.c_void_p), r[9],
                        r[12], r[13], r[10], r[11], P(org), P(d))
        assert np.array_equal(org, o[:3]) and np.array_equal(d, o[3:])


@pytest.mark.parametrize("kind", ["sphere", "plane"])
def test_sphere_plane_kat(kat, kind):
    fn = getattr(po.lib(), "xo_kat_" + kind)
    for r, o in zip(kat[kind + "_in"], kat[kind + "_out"]):
        out = np.zeros(7)
        h = fn(P(r[:4]), P(r[4:7]), P(r[7:10]), P(out))
        assert h == o[0]
        if h:
            assert np.array_equal(out, o[1:])


def test_triangle_kat(kat):
    L = po.lib()
    for r, o in zip(kat["triangle_in"], kat["triangle_out"]):
        out = np.zeros(7)
        h = L.xo_kat_triangle(P(r[:9]), P(r[9:18]), P(r[18:21]), P(r[21:24]), P(out))
        assert h == o[0]
        if h:
            assert np.array_equal(out, o[1:])


def test_aabb_kat(kat):
    L = po.lib()
    got = [L.xo_kat_aabb(P(r[0:3]), P(r[3:6]), P(r[6:9]), P(r[9:12])) for r in kat["aabb_in"]]
    assert np.array_equal(np.array(got), kat["aabb_out"])


def test_sampling_kat(kat):
    """hemisphere / diffuse / lobe consume the same libc rand() values as the
    reference and return the same bits (sample.inl:28-107)."""
    L = po.lib()
    tab = kat["rand_table"].astype(np.int32)
    rm = int(kat["rand_max"])
    for i in range(tab.shape[0]):
        out = np.zeros(3)
        L.xo_kat_hemisphere(P(tab[i]), rm, P(kat["hemisphere_n"][i]), P(out))
        assert np.array_equal(out, kat["hemisphere_out"][i])
        L.xo_kat_diffuse(P(tab[i]), rm, P(kat["hemisphere_n"][i]), P(out))
        assert np.array_equal(out, kat["diffuse_out"][i])
        L.xo_kat_lobe(P(tab[i]), rm, P(kat["hemisphere_n"][i]), P(kat["lobe_d"][i]), kat["lobe_e"][i], P(out))
        assert np.array_equal(out, kat["lobe_out"][i])


def test_material_kat(kat):
    L = po.lib()
    tab = kat["rand_table"].astype(np.int32)
    rm = int(kat["rand_max"])
    for i, (r, o) in enumerate(zip(kat["material_in"], kat["material_out"])):
        m = po.XoMaterial()
        m.type = int(r[0]); m.diffuse[:] = list(r[2:5]); m.specular[:] = list(r[5:8])
        m.emissive[:] = list(r[8:11]); m.reflectance = r[11]; m.exponent = r[12]
        out = np.zeros(9)
        cont = L.xo_kat_material(C.byref(m), P(tab[i]), rm, P(r[13:16]), P(r[16:19]), P(r[19:22]), P(out))
        assert cont == o[0]
        assert np.array_equal(out[6:], o[7:])
        if cont:
            assert np.array_equal(out[:6], o[1:7])


def test_gradient_kat(kat):
    L = po.lib()
    for r, o in zip(kat["gradient_in"], kat["gradient_out"]):
        a = (C.c_float * 3)(*r[0:3]); b = (C.c_float * 3)(*r[3:6]); out = np.zeros(3, np.float32)
        L.xo_kat_gradient(C.cast(a, C.c_void_p), C.cast(b, C.c_void_p), P(r[6:9]), P(out))
        assert np.array_equal(out.astype(np.float64), o)


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k"])
@pytest.mark.parametrize("accel", [po.XO_ACCEL_OCTREE, po.XO_ACCEL_BVH])
def test_primary_hits_golden(name, accel):
    """Closest hit, object, triangle index (octree item), t, point and normal of
    every primary ray equal the reference's (scene.cc:191-216, octree.tml:206-249)."""
    spec, w, h = small_scenes()[name]
    g = np.load(os.path.join(GOLD, "hits_%s.npz" % name))
    assert list(g["names"]) == ["o%05d" % i for i in range(len(spec.obj_kind))]
    sc = po.OracleScene(spec, accel)
    org, d = po.camera_rays(spec, w, h, g["xy"])
    assert np.array_equal(org, g["org"]) and np.array_equal(d, g["dir"])
    r = sc.trace(org, d)
    m = g["hit"] == 1
    assert np.array_equal(r["hit"], g["hit"])
    assert np.array_equal(r["t"][m], g["t"][m])
    assert np.array_equal(r["obj"][m], g["obj"][m])
    assert np.array_equal(r["point"][m], g["point"][m])
    assert np.array_equal(r["normal"][m], g["normal"][m])
    if spec.n_tris:
        pm = m & (g["prim"] >= 0)
        assert np.array_equal(r["prim"][pm] - spec.obj_first[r["obj"][pm]], g["prim"][pm])


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k"])
@pytest.mark.parametrize("integ", ["stencil", "depth"])
def test_deterministic_frames_golden(name, integ):
    spec, w, h = small_scenes()[name]
    g = np.load(os.path.join(GOLD, "render_%s.npz" % name))
    sc = po.OracleScene(spec, po.XO_ACCEL_OCTREE)
    kind = po.STENCIL if integ == "stencil" else po.DEPTH
    img, rays = sc.render(kind, w, h, spp=int(g[integ + "_spp"]), pixels=g[integ + "_xy"])
    assert np.array_equal(img, g[integ + "_rgba"])
    assert rays == w * h * int(g[integ + "_spp"])


def _rmse(a, b):
    return float(np.sqrt(np.mean((a[:, :3] - b[:, :3]) ** 2)))


def stochastic_agreement(O, R):
    """Leave-one-out comparison: the oracle frame against the mean of 3 reference
    frames, next to each reference frame against the mean of the other 3."""
    n = R.shape[0]
    ref = np.mean([_rmse(R[i], R[[j for j in range(n) if j != i]].mean(0)) for i in range(n)])
    got = np.mean([_rmse(O, R[[j for j in range(n) if j != i]].mean(0)) for i in range(n)])
    return got, ref


@pytest.mark.parametrize("name,key,integ,md", [
    ("spheres64", "ao100", po.AO, 100.0), ("spheres64", "ao0.2", po.AO, 0.2),
    ("terrain20k", "ao100", po.AO, 100.0), ("terrain20k", "ao0.2", po.AO, 0.2),
    ("hairball20k", "ao100", po.AO, 100.0), ("hairball20k", "ao0.2", po.AO, 0.2),
    ("spheres64", "pt", po.PATHTRACER, 100.0)])
def test_stochastic_frames_within_reference_noise(name, key, integ, md):
    spec, w, h = small_scenes()[name]
    g = np.load(os.path.join(GOLD, "render_%s.npz" % name))
    sc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    O, rays = sc.render(integ, w, h, spp=int(g[key + "_spp"]), rdepth=4, ao_max_distance=md, seed=777,
                        pixels=g[key + "_xy"])
    R = g[key + "_rgba"]
    got, ref = stochastic_agreement(O, R)
    assert got <= 1.25 * ref + 1e-6, (got, ref)
    # No bias in the frame mean beyond 4.5 standard errors.  The standard error
    # comes from the per-pixel variance between the reference frames (one
    # channel: AO writes the same value to r, g and b); O - mean(R) has variance
    # se^2 (1 + 1/n).
    n = R.shape[0]
    for ch in range(3):
        diff = O[:, ch] - R[:, :, ch].mean(0)
        se = np.sqrt(R[:, :, ch].var(0, ddof=1).mean() / diff.size * (1 + 1.0 / n))
        assert abs(diff.mean()) < 4.5 * se + 1e-5, (ch, diff.mean(), se)
    if key == "pt":
        ref_rays = [int(g["pt_rays_seed%d" % s]) for s in (21, 22, 23, 24)]
        assert abs(rays - np.mean(ref_rays)) < 5 * np.std(ref_rays) + 0.005 * np.mean(ref_rays)


def test_stream_rng_is_uniform():
    """The counter stream (SplitMix64 finaliser) shared with the GPU path."""
    k = po.path_key(1234, 99)
    u = np.array([po.stream_uniform(k, i) for i in range(20000)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.01
    assert abs(u.var() - 1 / 12) < 0.005
    assert np.all(u * 16777216.0 == np.floor(u * 16777216.0))


def _primary_scene(name):
    return {"spheres64": lambda: scenes.spheres_scene(64, seed=1, name="spheres64"),
            "terrain20k": lambda: scenes.terrain_scene(20_000, seed=2, name="terrain20k"),
            "uvscene": lambda: scenes.uv_scene(6)}[name]()


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "uvscene"])
@pytest.mark.parametrize("integ,code", [("normal", po.NORMAL), ("uv", po.UV), ("emission", po.EMISSION),
                                        ("wireframe", po.WIREFRAME)])
def test_primary_integrators_golden(name, integ, code):
    """normal, uv, emission and wireframe integrators (normal/uv/emission/
    wireframe integrator.cc): the restatement reproduces the reference's frames
    bit for bit, texture coordinates of spheres, planes (with u/v scales) and
    OBJ-textured triangles included."""
    g = np.load(os.path.join(GOLD, "render_primary_%s.npz" % name))
    spec = _primary_scene(name)
    orc = po.OracleScene(spec, po.XO_ACCEL_OCTREE)
    xy = g["%s_xy" % integ]
    out, rays = orc.render(code, int(g["width"]), int(g["height"]), spp=int(g["spp"]), pixels=xy)
    ref = g["%s_rgba" % integ]
    assert rays == int(g["%s_rays" % integ])
    # a u/v scale below 1 drives asin out of its domain on spheres: the
    # reference writes NaN there, and so must the restatement
    assert np.array_equal(out, ref, equal_nan=True), np.nanmax(np.abs(out - ref))


def _f3(v):
    return np.ascontiguousarray(v, np.float32).ctypes.data_as(C.c_void_p)


def test_camera_kat_erp_ods_cubemap_dof():
    """ERP, ODS, cubemap and thin-lens depth-of-field rays (camera/*.cc),
    including the Matrix4x4f euler rotation and the two prng_c lens draws,
    bit for bit against the reference."""
    k = np.load(os.path.join(GOLD, "kat_cameras.npz"))
    L = po.lib()
    o, d = np.zeros(3), np.zeros(3)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    for kind in ("erp", "ods"):
        for r, want in zip(k[kind + "_in"], k[kind + "_out"]):
            if kind == "erp":
                L.xo_kat_camera_erp(_f3(r[0:3]), _f3(r[3:6]), r[9], r[10], r[7], r[8], P(o), P(d))
            else:
                L.xo_kat_camera_ods(_f3(r[0:3]), _f3(r[3:6]), r[6], r[9], r[10], r[7], r[8], P(o), P(d))
            assert np.array_equal(np.concatenate([o, d]), want), (kind, r)
    for r, want in zip(k["cubemap_in"], k["cubemap_out"]):
        L.xo_kat_camera_cubemap(_f3(r[0:3]), r[5], r[6], r[3], r[4], P(o), P(d))
        assert np.array_equal(np.concatenate([o, d]), want), ("cubemap", r)
    for r, tab, want in zip(k["dof_in"], k["dof_table"], k["dof_out"]):
        t = np.ascontiguousarray(tab, np.int32)
        L.xo_kat_camera_dof(P(t), int(k["rand_max"]), _f3(r[1:4]), _f3(r[4:7]), _f3(r[7:10]), r[10], r[11], r[12],
                            r[15], r[16], r[13], r[14], P(o), P(d))
        assert np.array_equal(np.concatenate([o, d]), want), ("dof", r)


def _camera_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.camera_cases()


@pytest.mark.parametrize("case", range(4))
def test_camera_frames_with_grid_antialiasing_golden(case):
    """Stencil, depth and normal frames through the perspective (aa 3), ERP,
    ODS and cubemap (aa 2) cameras: grid positions, weights 1/(aa^2 spp) and
    per-sample folds equal the reference's frames bit for bit."""
    g = np.load(os.path.join(GOLD, "render_cameras.npz"))
    tag, cam, w, h, aa = _camera_cases()[case]
    spec = scenes.spheres_scene(64, seed=1, name="cam_" + tag, camera=cam)
    orc = po.OracleScene(spec, po.XO_ACCEL_OCTREE)
    for integ, code in (("stencil", po.STENCIL), ("depth", po.DEPTH), ("normal", po.NORMAL)):
        xy = g["%s_%s_xy" % (tag, integ)]
        out, rays = orc.render(code, w, h, spp=2, pixels=xy, aa=aa)
        assert rays == int(g["%s_%s_rays" % (tag, integ)])
        ref = g["%s_%s_rgba" % (tag, integ)]
        assert np.array_equal(out, ref, equal_nan=True), (tag, integ, np.nanmax(np.abs(out - ref)))


def _kat_textures(k):
    """The sampler fixtures' textures as the reference holds them after
    loading: texels and ctypes layout rows (one texel array per texture)."""
    out = []
    i = 0
    while "tex%d_pixels" % i in k:
        filt, fx, fy = (int(v) for v in k["tex%d_mode" % i])
        t = scenes.Texture(k["tex%d_pixels" % i], filt, bool(fx), bool(fy))
        tx = t.texels()
        out.append((po.texture_structs(np.array([[tx.shape[1], tx.shape[0], filt, 0]])), tx))
        i += 1
    return out


def test_texture_sampler_kat():
    """Texture2D::sample with nearest and bilinear filtering, flips, RGB and
    RGBA textures of odd sizes, texcoords outside [0, 1], NaN and infinities
    (sampler_tex.cc:37-45, nimg/sample.cc:8-52): bit for bit."""
    k = np.load(os.path.join(GOLD, "kat_textures.npz"))
    texs = _kat_textures(k)
    L = po.lib()
    out = (C.c_float * 3)()
    for (i, u, v), want in zip(k["tex_in"], k["tex_out"]):
        st, tx = texs[int(i)]
        L.xo_kat_texture(C.cast(st, C.c_void_p), P(tx), float(u), float(v), out)
        assert np.array_equal(np.float32(out), want, equal_nan=True), (int(i), u, v, list(out), want)


def test_erp_and_cubemap_sampler_kat():
    """ERP::sample and Cubemap::sample (sampler_erp.cc:13-26,
    sampler_cubemap.cc:13-36) on random, axis-aligned, zero and NaN
    directions: bit for bit."""
    k = np.load(os.path.join(GOLD, "kat_textures.npz"))
    L = po.lib()
    etx = scenes.Texture(k["erp_pixels"]).texels()
    est = po.texture_structs(np.array([[etx.shape[1], etx.shape[0], 0, 0]]))
    ftx = [scenes.Texture(k["face%d_pixels" % f]).texels() for f in range(6)]
    offs = np.cumsum([0] + [t.shape[0] * t.shape[1] for t in ftx])[:-1]
    fst = po.texture_structs(np.array([[t.shape[1], t.shape[0], 0, o] for t, o in zip(ftx, offs)]))
    fall = np.ascontiguousarray(np.concatenate([t.reshape(-1, 4) for t in ftx]))
    out = (C.c_float * 3)()
    for d, we, wc in zip(k["dirs"], k["erp_out"], k["cube_out"]):
        dv = np.ascontiguousarray(d, np.float64)
        L.xo_kat_erp(C.cast(est, C.c_void_p), P(etx), P(dv), out)
        assert np.array_equal(np.float32(out), we, equal_nan=True), ("erp", d)
        L.xo_kat_cubemap(C.cast(fst, C.c_void_p), P(fall), P(dv), out)
        assert np.array_equal(np.float32(out), wc, equal_nan=True), ("cubemap", d)


@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_frames_golden(env):
    """Textured scenes through the reference's own loader (PNG files,
    filtering and flip keys): the emission frame (aa 2) folds each sample's
    emissive texel, and the depth-1 pathtracer frame is the environment's texel
    on a miss and the emissive sampler's on an emissive hit.  Bit for bit."""
    import importlib.util
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    w, h = mg.texture_frame_size()
    g = np.load(os.path.join(GOLD, "render_textures.npz"))
    spec = scenes.textured_scene(env)
    orc = po.OracleScene(spec, po.XO_ACCEL_OCTREE)
    for integ, code, spp, rdepth, aa in (("emission", po.EMISSION, 2, 1, 2), ("pathtracer", po.PATHTRACER, 2, 1, 1)):
        xy = g["%s_%s_xy" % (env, integ)]
        out, rays = orc.render(code, w, h, spp=spp, rdepth=rdepth, pixels=xy, aa=aa)
        assert rays == int(g["%s_%s_rays" % (env, integ)])
        ref = g["%s_%s_rgba" % (env, integ)]
        assert np.array_equal(out, ref, equal_nan=True), (env, integ, np.nanmax(np.abs(out - ref)))


@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_pathtracer_within_reference_noise(env):
    """Depth-4 paths over textured diffuse, specular and emissive samplers:
    within the reference's noise (four reference seeds)."""
    g = np.load(os.path.join(GOLD, "render_textures.npz"))
    spec = scenes.textured_scene(env)
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    w, h = 64, 48
    O, _ = orc.render(po.PATHTRACER, w, h, spp=16, rdepth=4, seed=777, pixels=g["%s_pt_xy" % env])
    R = g["%s_pt_rgba" % env]
    got, ref = stochastic_agreement(O, R)
    assert got <= 1.25 * ref + 1e-6, (got, ref)
    n = R.shape[0]
    for ch in range(3):
        diff = O[:, ch] - R[:, :, ch].mean(0)
        se = np.sqrt(R[:, :, ch].var(0, ddof=1).mean() / diff.size * (1 + 1.0 / n))
        assert abs(diff.mean()) < 4.5 * se + 1e-5, (ch, diff.mean(), se)


def test_raygraph_golden():
    """The depth integrator's raygraph (depth/integrator.cc:43-51) exported as
    the GUI does (render::assemble, raygraph::write): the oracle's records,
    listed in the reference's tile and produce order and printed as an ostream
    prints them, give the reference's PLY byte for byte."""
    import importlib.util
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    spec, w, h, spp, aa = mg.raygraph_case()
    g = np.load(os.path.join(GOLD, "raygraph.npz"))
    orc = po.OracleScene(spec, po.XO_ACCEL_OCTREE)
    out, rec = orc.render_raygraph(w, h, spp=spp, aa=aa, pixels=po.raygraph_pixel_order(w, h))
    assert po.raygraph_ply(rec) == g["ply"].tobytes().decode()


def test_obj_mtl_frames_golden():
    """Meshes loaded from an OBJ with an MTL library (parseutil.cc:588-682):
    the shapes come last in the scene's object map, BlinnPhong materials carry
    Kd / Ks or map_Kd / map_Ks, Emissive ones Ke or map_Ke, textures flipped
    horizontally (create_sampler); the generator's description of that scene
    renders the reference's depth, uv, emission and depth-1 pathtracer frames
    bit for bit, and depth-4 paths within its noise."""
    g = np.load(os.path.join(GOLD, "render_mtl.npz"))
    spec = scenes.mtl_scene()
    orc = po.OracleScene(spec, po.XO_ACCEL_OCTREE)
    for integ, code in (("depth", po.DEPTH), ("uv", po.UV), ("emission", po.EMISSION), ("pathtracer", po.PATHTRACER)):
        out, rays = orc.render(code, 64, 48, spp=2, rdepth=1, pixels=g["%s_xy" % integ])
        assert rays == int(g["%s_rays" % integ])
        assert np.array_equal(out, g["%s_rgba" % integ], equal_nan=True), integ
    O, _ = po.OracleScene(spec, po.XO_ACCEL_BVH).render(po.PATHTRACER, 64, 48, spp=16, rdepth=4, seed=777,
                                                        pixels=g["pt_xy"])
    got, ref = stochastic_agreement(O, g["pt_rgba"])
    assert got <= 1.25 * ref + 1e-6, (got, ref)


def test_random_distribution_within_reference_noise():
    """The random sample distribution (aa.cc:34-48): aa positions per pixel,
    each taken spp times at weight 1/(aa spp).  The reference draws the jitter
    offsets from rand(); the oracle from a stream keyed by (seed, position,
    pixel).  Rays traced are equal, stencil coverage takes the same multiples
    of 1/aa, and stencil and depth frames agree within the noise of four
    seeds on each side."""
    import importlib.util
    from tests.parity import random_distribution_agreement
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    cam, w, h, spp, cases, seeds = mg.random_case()
    g = np.load(os.path.join(GOLD, "render_random.npz"))
    orc = po.OracleScene(scenes.spheres_scene(64, seed=1, name="cam_random", camera=cam), po.XO_ACCEL_BVH)
    for integ, aa in cases:
        key = "%s_aa%d" % (integ, aa)
        code = po.STENCIL if integ == "stencil" else po.DEPTH
        O = []
        for s, ref_rays in zip(seeds, g[key + "_rays"]):
            o, rays = orc.render(code, w, h, spp=spp, seed=s, pixels=g[key + "_xy"], aa=aa,
                                 distribution=po.SAMPLES_RANDOM)
            assert rays == int(ref_rays) == w * h * aa * spp
            O.append(o)
        random_distribution_agreement(g[key + "_rgba"], np.stack(O), 3 if integ == "stencil" else 0,
                                      aa if integ == "stencil" else None)


def test_lobe_edge_kat():
    """sample::lobe (sample.inl:61-90) at its edges: the direction along the
    normal (the frame stays the identity), 1 - d.n just below and above 1e-8,
    exponents up to 2000 where pow(vdotr, e) underflows and the result is the
    zero or unnormalised vector: the oracle returns the reference's bits."""
    g = np.load(os.path.join(GOLD, "render_phong.npz"))
    L = po.lib()
    rm = int(g["rand_max"])
    zero = 0
    for i in range(g["lobe_out"].shape[0]):
        tab = np.ascontiguousarray(g["lobe_rand"][i], np.int32)
        out = np.zeros(3)
        L.xo_kat_lobe(P(tab), rm, P(g["lobe_n"][i]), P(g["lobe_d"][i]), float(g["lobe_e"][i]), P(out))
        assert np.array_equal(out, g["lobe_out"][i]), (i, out, g["lobe_out"][i])
        zero += int(np.dot(out, out) == 0.0)
    assert zero >= 4   # the identity-frame rows that give no direction are covered


def test_phong_pathtracer_within_reference_noise():
    """Phong and Blinn-Phong paths (render_phong.npz, four reference seeds):
    the oracle's frames have per-pixel RMSE against the 4096-spp render within
    the reference's at 16 spp, and the centre pixel (a head-on hit, identity
    lobe frame) agrees with the reference's to within its noise."""
    from tests import parity
    g = np.load(os.path.join(GOLD, "render_phong.npz"))
    t = np.load(os.path.join(GOLD, "truth.npz"))
    xy, truth = t["phong_pt_xy"], t["phong_pt_rgba"]
    assert np.array_equal(xy, g["pt_xy"])
    spec = scenes.phong_scene()
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    frames, rays = [], []
    for seed in (777, 778):
        o, r = orc.render(po.PATHTRACER, int(g["width"]), int(g["height"]), spp=int(g["spp"]),
                          rdepth=int(g["depth"]), seed=seed, pixels=xy)
        frames.append(o)
        rays.append(r)
    R = g["pt_rgba"]
    parity.converged_rmse_bar(np.stack(frames), truth, [parity.rmse(r, truth) for r in R], "oracle phong")
    ref_rays = g["pt_rays"].astype(np.float64)
    assert abs(np.mean(rays) - ref_rays.mean()) <= 5 * ref_rays.std() + 0.005 * ref_rays.mean()
    c = np.nonzero((xy[:, 0] == int(g["width"]) // 2) & (xy[:, 1] == int(g["height"]) // 2))[0][0]
    rc = R[:, c, :3].astype(np.float64)
    oc = np.stack(frames)[:, c, :3].astype(np.float64)
    assert np.all(np.abs(oc.mean(0) - rc.mean(0)) <= 4.5 * np.sqrt(rc.var(0, ddof=1) / 4 + oc.var(0, ddof=1) / 2)
                  + 1e-3), (oc, rc)
