"""GPU parity: the CUDA path through the C ABI against the oracle restatement
and the reference's own golden fixtures.

Bars (from the hot-path contract):
* LBVH integer steps (Morton codes, sort order, Karras topology): bit-exact
  against the CPU re-implementation (oracle/lbvh_cpu.c).
* Primary hits: primitive agreement >= 99.99% of pixels, every disagreement
  explained as a tie (|dt|/t <= 1e-5 between the two primitives in FP64) or a
  grazing hit (barycentric margin or sphere discriminant below 1e-5); relative
  depth error <= 1e-5 where the primitives agree.
* Stencil frames identical where hits agree; depth frames within 1e-5 relative.
* AO / pathtracer: per-pixel RMSE against the reference's frames within the
  reference's own sampling noise at equal spp.
* 8-bit quantised BVH: the same hits as the FP32 BVH.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests import parity
from xtracer_b200 import scenes, xtgpu

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


def small_scenes():
    return {"spheres64": (scenes.spheres_scene(64, seed=1, name="spheres64"), 64, 64),
            "terrain20k": (scenes.terrain_scene(20_000, seed=2, name="terrain20k"), 96, 54),
            "hairball20k": (scenes.hairball_scene(20_000, seed=3, name="hairball20k"), 64, 64)}


def lbvh_cpu(spec):
    L = po.lib()
    L.xo_lbvh_build.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p] + [C.c_void_p] * 4
    n = spec.n_tris + spec.spheres.shape[0]
    keys = np.zeros(max(n, 1), np.uint32); order = np.zeros(max(n, 1), np.uint32)
    left = np.zeros(max(n - 1, 1), np.int32); right = np.zeros(max(n - 1, 1), np.int32)
    tris = np.ascontiguousarray(spec.tris.reshape(-1), np.float32)
    sph = np.ascontiguousarray(spec.spheres.reshape(-1), np.float32)
    L.xo_lbvh_build(spec.n_tris, tris.ctypes.data_as(C.c_void_p), spec.spheres.shape[0],
                    sph.ctypes.data_as(C.c_void_p), *[a.ctypes.data_as(C.c_void_p) for a in (keys, order, left, right)])
    return keys[:n], order[:n], left[:max(n - 1, 0)], right[:max(n - 1, 0)]


def ploc_cpu(spec):
    L = po.lib()
    L.xo_ploc_build.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p] + [C.c_void_p] * 4
    n = spec.n_tris + spec.spheres.shape[0]
    keys = np.zeros(max(n, 1), np.uint32); order = np.zeros(max(n, 1), np.uint32)
    left = np.zeros(max(n - 1, 1), np.int32); right = np.zeros(max(n - 1, 1), np.int32)
    tris = np.ascontiguousarray(spec.tris.reshape(-1), np.float32)
    sph = np.ascontiguousarray(spec.spheres.reshape(-1), np.float32)
    assert L.xo_ploc_build(spec.n_tris, tris.ctypes.data_as(C.c_void_p), spec.spheres.shape[0],
                           sph.ctypes.data_as(C.c_void_p),
                           *[a.ctypes.data_as(C.c_void_p) for a in (keys, order, left, right)]) == 0
    return keys[:n], order[:n], left[:max(n - 1, 0)], right[:max(n - 1, 0)]


def with_builder(builder):
    """Sets the process-wide BVH builder for scenes created inside; restores it."""
    import contextlib

    @contextlib.contextmanager
    def ctx():
        keep = xtgpu.get_tuning().bvh_builder
        xtgpu.set_tuning(bvh_builder=builder)
        try:
            yield
        finally:
            xtgpu.set_tuning(bvh_builder=keep)
    return ctx()


def duplicate_scene():
    """Many triangles with identical centroids: equal Morton codes everywhere."""
    t = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)
    tris = np.repeat(t, 1000, axis=0)
    tris[500:] += np.float32(4.0)
    spec = scenes.terrain_scene(8, seed=1, name="dup")
    spec.tris = tris
    spec.obj_count = np.array([tris.shape[0]], np.int32)
    spec.mesh_obj = None
    return spec


def tiny_scene(n_spheres):
    return scenes.spheres_scene(n_spheres, seed=9, name="tiny%d" % n_spheres, with_light=False)


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k", "dup", "tiny1", "tiny2", "tiny3",
                                  "hairball300k"])
def test_lbvh_bit_exact_vs_cpu(name):
    if name in small_scenes():
        spec = small_scenes()[name][0]
    elif name == "dup":
        spec = duplicate_scene()
    elif name == "hairball300k":
        spec = scenes.hairball_scene(300_000, seed=5)
    else:
        spec = tiny_scene(int(name[-1]))
    with with_builder(0):
        sc = xtgpu.Scene(spec)
    ex = sc.bvh_export()
    keys, order, left, right = lbvh_cpu(spec)
    assert np.array_equal(ex["morton"], keys)
    assert np.array_equal(ex["order"], order)
    assert np.array_equal(ex["left"], left)
    assert np.array_equal(ex["right"], right)
    n = keys.size
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    if n > 1:
        # every node but the root has exactly one parent
        inner = np.concatenate([left[left >= 0], right[right >= 0]])
        leaves = np.concatenate([~left[left < 0], ~right[right < 0]])
        assert np.array_equal(np.sort(inner), np.arange(1, n - 1))
        assert np.array_equal(np.sort(leaves), np.arange(n))
    sc.close()


def gpu_primary(spec, w, h, fmt=xtgpu.NODES_FP32, sc=None, px=None):
    """Primary rays through the GPU: the FP64 reference camera rays rounded to
    FP32, traced by xtgpu_trace_host.  px: (x, y) pixel list (default: the
    frame in row-major order)."""
    if px is None:
        ys, xs = np.mgrid[0:h, 0:w]
        px = np.stack([xs.ravel(), ys.ravel()], 1)
    org, dirs = po.camera_rays(spec, w, h, px)
    own = sc is None
    if own:
        sc = xtgpu.Scene(spec, node_formats=(fmt,))
    hits = sc.intersection(org.astype(np.float32), dirs.astype(np.float32), node_format=fmt)
    if own:
        sc.close()
    return org, dirs, hits


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k"])
@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8])
def test_primary_hits_vs_reference_golden(name, fmt):
    spec, w, h = small_scenes()[name]
    g = np.load(os.path.join(GOLD, "hits_%s.npz" % name))
    # fixture records are in the reference driver's tile order
    org, dirs, hits = gpu_primary(spec, w, h, fmt, px=g["xy"])
    assert np.array_equal(org, g["org"]) and np.array_equal(dirs, g["dir"])
    g_hit = (hits["prim"] != 0xffffffff).astype(np.int32)
    g_gid = hits["prim"].astype(np.int64)
    r_hit = g["hit"].astype(np.int32)
    r_gid = np.array([parity.global_prim(spec, o, p) if o >= 0 else -1 for o, p in zip(g["obj"], g["prim"])])
    n_agree, tie, graze, bad = parity.classify(spec, org, dirs, g_hit, g_gid, hits["t"].astype(np.float64),
                                               r_hit, r_gid, g["t"])
    print("[%s fmt %d] primitive agreement %.6f of %d rays (%d ties, %d grazing)" %
          (name, fmt, n_agree / g_hit.size, g_hit.size, tie, graze))
    assert not bad, "unexplained disagreements at %s" % bad[:10]
    assert n_agree >= 0.9999 * g_hit.size
    m = (g_hit == 1) & (r_hit == 1) & (g_gid == r_gid)
    rel = np.abs(hits["t"][m].astype(np.float64) - g["t"][m]) / g["t"][m]
    assert rel.max() <= 1e-5, rel.max()


def test_primary_hits_terrain_200k_vs_oracle():
    """A larger mesh than the fixtures, checked against the oracle restatement."""
    spec = scenes.terrain_scene(200_000, seed=11)
    w, h = 480, 270
    org, dirs, hits = gpu_primary(spec, w, h)
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    r = orc.trace(org, dirs)
    r_gid = parity.oracle_global_prim(spec, r["obj"], r["prim"])
    g_hit = (hits["prim"] != 0xffffffff).astype(np.int32)
    g_gid = hits["prim"].astype(np.int64)
    n_agree, tie, graze, bad = parity.classify(spec, org, dirs, g_hit, g_gid, hits["t"].astype(np.float64),
                                               r["hit"], r_gid, r["t"])
    assert not bad, "unexplained disagreements: %d" % len(bad)
    assert n_agree >= 0.9999 * g_hit.size
    m = (g_hit == 1) & (r["hit"] == 1) & (g_gid == r_gid)
    rel = np.abs(hits["t"][m].astype(np.float64) - r["t"][m]) / r["t"][m]
    assert rel.max() <= 1e-5, rel.max()


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k", "dup", "tiny2", "tiny3",
                                  "hairball300k"])
def test_ploc_bit_exact_vs_cpu(name):
    """The PLOC hierarchy (bvh_builder 1): clustering, node numbering and the
    depth-first leaf order equal the CPU re-implementation bit for bit."""
    if name in small_scenes():
        spec = small_scenes()[name][0]
    elif name == "dup":
        spec = duplicate_scene()
    elif name == "hairball300k":
        spec = scenes.hairball_scene(300_000, seed=5)
    else:
        spec = tiny_scene(int(name[-1]))
    with with_builder(1):
        sc = xtgpu.Scene(spec)
        ex = sc.bvh_export()
        sc.close()
    keys, order, left, right = ploc_cpu(spec)
    assert np.array_equal(ex["order"], order)
    assert np.array_equal(ex["morton"], keys)
    assert np.array_equal(ex["left"], left)
    assert np.array_equal(ex["right"], right)


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k"])
@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8])
def test_ploc_tree_gives_the_same_hits(name, fmt):
    """Any hierarchy gives the same closest hits (ties go to the lower
    primitive id): PLOC and LBVH frames are equal bit for bit."""
    spec, w, h = small_scenes()[name]
    a = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    with with_builder(1):
        b = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    for integ in (xtgpu.DEPTH, xtgpu.PATHTRACER):
        ia, ra = a.render(integ, w, h, spp=4, rdepth=4, seed=8, node_format=fmt)
        ib, rb = b.render(integ, w, h, spp=4, rdepth=4, seed=8, node_format=fmt)
        assert ra == rb and np.array_equal(ia, ib)
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k"])
def test_q8_hits_equal_fp32(name):
    spec, w, h = small_scenes()[name]
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8))
    _, _, a = gpu_primary(spec, w, h, xtgpu.NODES_FP32, sc)
    _, _, b = gpu_primary(spec, w, h, xtgpu.NODES_Q8, sc)
    same = (a["prim"] == b["prim"]) & ((a["t"] == b["t"]) | (a["prim"] == 0xffffffff))
    assert same.mean() >= 0.9999
    sc.close()


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k", "dup", "tiny1", "tiny2", "tiny3"])
@pytest.mark.parametrize("leaf", [1, 2, 3])
@pytest.mark.parametrize("collapse", [0, 1])
def test_w8_hits_equal_fp32(name, leaf, collapse):
    """The 8-wide quantised BVH, collapsed greedily (0) or by surface-area
    cost with subtrees of up to 3 primitives as leaves (1), finds the same
    closest hits as the binary FP32 BVH, bit for bit: conservative boxes, the
    same primitive tests, and ties broken by primitive id whatever the visiting
    order."""
    if name in small_scenes():
        spec, w, h = small_scenes()[name]
    else:
        spec = duplicate_scene() if name == "dup" else tiny_scene(int(name[-1]))
        w, h = 48, 32
    keep = xtgpu.get_tuning().wide_collapse
    try:
        xtgpu.set_tuning(wide_collapse=collapse)
        sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_W8), leaf_size=leaf)
    finally:
        xtgpu.set_tuning(wide_collapse=keep)
    assert sc.tuning().wide_collapse == collapse
    info = sc.bvh_export()["info"]
    assert info.node_bytes_w8 > 0 and info.depth_w8 >= 1
    org, dirs, a = gpu_primary(spec, w, h, xtgpu.NODES_FP32, sc)
    _, _, b = gpu_primary(spec, w, h, xtgpu.NODES_W8, sc)
    assert np.array_equal(a["prim"], b["prim"])
    assert np.array_equal(a["t"], b["t"])
    # secondary-like rays from inside the scene, in all directions
    rng = np.random.default_rng(leaf)
    lo = spec.tris.reshape(-1, 3).min(0) if spec.n_tris else spec.spheres[:, :3].min(0)
    hi = spec.tris.reshape(-1, 3).max(0) if spec.n_tris else spec.spheres[:, :3].max(0)
    o = (lo + (hi - lo) * rng.random((20000, 3))).astype(np.float32)
    d = rng.normal(size=(20000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    a = sc.intersection(o, d, node_format=xtgpu.NODES_FP32)
    b = sc.intersection(o, d, node_format=xtgpu.NODES_W8)
    assert np.array_equal(a["prim"], b["prim"])
    assert np.array_equal(a["t"], b["t"])
    sc.close()


@pytest.mark.parametrize("variant,refill,steps", [(0, 8, 8), (1, 8, 8), (2, 8, 1), (2, 16, 8), (2, 32, 64)])
@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8])
def test_extend_variants_agree(variant, refill, steps, fmt):
    """Every extend kernel (warp-batched, per-step refill, pooled lanes with a
    vote every few steps) and node format returns the same hits."""
    spec, w, h = small_scenes()["hairball20k"]
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8), leaf_size=1)
    rng = np.random.default_rng(7)
    o = (rng.random((50000, 3)) * 2.4 - 1.2).astype(np.float32)
    d = rng.normal(size=(50000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    ref = sc.intersection(o, d, node_format=xtgpu.NODES_FP32)
    keep = {k: getattr(xtgpu.get_tuning(), k) for k, _ in xtgpu.Tuning._fields_}
    try:
        xtgpu.set_tuning(extend_variant=variant, refill_threshold=refill, steps_per_vote=steps)
        got = sc.intersection(o, d, node_format=fmt)
    finally:
        xtgpu.set_tuning(**keep)
    sc.close()
    assert np.array_equal(ref["prim"], got["prim"])
    assert np.array_equal(ref["t"], got["t"])


@pytest.mark.parametrize("pf,pv", [(xtgpu.NODES_FP32, 0), (xtgpu.NODES_W8, 0), (xtgpu.NODES_Q8, 2)])
def test_primary_pass_format_keeps_frames(pf, pv):
    """The camera rays may take another node format and extend kernel than the
    bounce rays; every format and kernel returns the same hits, so the frames
    are the same bit for bit."""
    spec, w, h = small_scenes()["hairball20k"]
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8), leaf_size=1)
    ref, rr = sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=9, node_format=xtgpu.NODES_W8)
    keep = {k: getattr(xtgpu.get_tuning(), k) for k, _ in xtgpu.Tuning._fields_}
    try:
        xtgpu.set_tuning(primary_node_format=pf, primary_variant=pv)
        got, rg = sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=9, node_format=xtgpu.NODES_W8)
    finally:
        xtgpu.set_tuning(**keep)
    sc.close()
    assert rr == rg
    assert np.array_equal(ref, got)


@pytest.mark.parametrize("integ", [xtgpu.STENCIL, xtgpu.DEPTH, xtgpu.AO, xtgpu.PATHTRACER])
def test_w8_frames_equal_fp32(integ):
    spec, w, h = small_scenes()["terrain20k"]
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_W8), leaf_size=1)
    a, ra = sc.render(integ, w, h, spp=8, rdepth=4, ao_max_distance=0.5, seed=4, node_format=xtgpu.NODES_FP32)
    b, rb = sc.render(integ, w, h, spp=8, rdepth=4, ao_max_distance=0.5, seed=4, node_format=xtgpu.NODES_W8)
    sc.close()
    assert ra == rb
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "hairball20k"])
def test_stencil_depth_frames_vs_reference_golden(name):
    """Stencil and depth frames (2 samples per pixel, each the pixel-centre
    ray) against the reference's, pixel by pixel: on every pixel whose primary
    ray hits the same primitive as the reference's (hits_*.npz), the stencil
    pixel is equal and the depth pixel gives the hit distance within 1e-5
    relative (depth = 1/ln t, so |1/depth_gpu - 1/depth_ref| = |ln t_gpu -
    ln t_ref| bounds the relative error of t); the primitive agrees on
    >= 99.99 % of pixels."""
    spec, w, h = small_scenes()[name]
    g = np.load(os.path.join(GOLD, "render_%s.npz" % name))
    hits_ref = np.load(os.path.join(GOLD, "hits_%s.npz" % name))
    sc = xtgpu.Scene(spec)
    # the primitive each pixel's ray meets, GPU and reference
    xy = hits_ref["xy"]
    _, _, gh = gpu_primary(spec, w, h, xtgpu.NODES_FP32, sc, px=xy)
    g_gid = np.where(gh["prim"] != 0xffffffff, gh["prim"].astype(np.int64), -1)
    r_gid = np.array([parity.global_prim(spec, o, p) if o >= 0 else -1
                      for o, p in zip(hits_ref["obj"], hits_ref["prim"])])
    agree_at = {tuple(p): bool(a) for p, a in zip(xy.tolist(), (g_gid == r_gid).tolist())}
    for key, integ in (("stencil", xtgpu.STENCIL), ("depth", xtgpu.DEPTH)):
        spp = int(g[key + "_spp"])
        img, rays = sc.render(integ, w, h, spp=spp)
        pxy = g[key + "_xy"]
        got = img[pxy[:, 1], pxy[:, 0]].astype(np.float64)
        ref = g[key + "_rgba"].astype(np.float64)
        same = np.array([agree_at[tuple(p)] for p in pxy.tolist()])
        print("[%s %s] primitive agrees on %.6f of %d pixels" % (name, key, same.mean(), same.size))
        assert same.mean() >= 0.9999
        if integ == xtgpu.STENCIL:
            assert np.array_equal(got[same], ref[same])
        else:
            hit = same & (ref[:, 3] > 0) & (ref[:, 0] != 0)
            assert np.array_equal(got[same & ~hit], ref[same & ~hit])
            dl = np.abs(1.0 / got[hit, 0] - 1.0 / ref[hit, 0])
            print("[%s depth] max |ln t_gpu - ln t_ref| %.3g over %d hit pixels" % (name, dl.max(), hit.sum()))
            assert dl.max() <= 1e-5, np.sort(dl)[-5:]
        assert rays == w * h * spp
    sc.close()


def _truth(name):
    t = np.load(os.path.join(GOLD, "truth.npz"))
    return t[name + "_xy"], t[name + "_rgba"]


@pytest.mark.parametrize("name,key,integ,md", [
    ("spheres64", "ao100", xtgpu.AO, 100.0), ("spheres64", "ao0.2", xtgpu.AO, 0.2),
    ("terrain20k", "ao100", xtgpu.AO, 100.0), ("terrain20k", "ao0.2", xtgpu.AO, 0.2),
    ("hairball20k", "ao100", xtgpu.AO, 100.0), ("hairball20k", "ao0.2", xtgpu.AO, 0.2),
    ("spheres64", "pt", xtgpu.PATHTRACER, 100.0)])
def test_stochastic_frames_within_reference_noise(name, key, integ, md):
    """Per-pixel RMSE against the 4096-spp render (truth.npz) within the
    reference's own at equal spp (its frames at four seeds, render_*.npz)."""
    spec, w, h = small_scenes()[name]
    g = np.load(os.path.join(GOLD, "render_%s.npz" % name))
    txy, truth = _truth("%s_%s" % (name, key))
    xy = g[key + "_xy"]
    assert np.array_equal(xy, txy)
    R = g[key + "_rgba"]
    sc = xtgpu.Scene(spec)
    frames = []
    for seed in (777, 778):
        img, rays = sc.render(integ, w, h, spp=int(g[key + "_spp"]), rdepth=4, ao_max_distance=md, seed=seed)
        frames.append(img[xy[:, 1], xy[:, 0]])
    sc.close()
    parity.converged_rmse_bar(np.stack(frames), truth, [parity.rmse(r, truth) for r in R], "%s %s" % (name, key))


@pytest.mark.parametrize("integ,md", [(xtgpu.AO, 0.5), (xtgpu.PATHTRACER, 100.0)])
def test_stochastic_same_stream_as_oracle(integ, md):
    """With the same random stream, GPU (FP32) and oracle (FP64) frames differ
    only where a rounding difference sends a path another way: at most a
    quarter of the sampling noise, and the rays traced within 1 %."""
    spec, w, h = small_scenes()["spheres64"]
    sc = xtgpu.Scene(spec)
    img, rays = sc.render(integ, w, h, spp=16, rdepth=4, ao_max_distance=md, seed=99)
    sc.close()
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    ys, xs = np.mgrid[0:h, 0:w]
    px = np.stack([xs.ravel(), ys.ravel()], 1)
    code = po.AO if integ == xtgpu.AO else po.PATHTRACER
    o, orays = orc.render(code, w, h, spp=16, rdepth=4, ao_max_distance=md, seed=99, pixels=px)
    o2, _ = orc.render(code, w, h, spp=16, rdepth=4, ao_max_distance=md, seed=100, pixels=px)
    parity.same_stream_bar(img, o, o2, "spheres64 %s" % ("ao" if integ == xtgpu.AO else "pt"))
    assert abs(rays - orays) <= 0.01 * orays


def _phong():
    return scenes.phong_scene(), 65, 49


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
def test_phong_pathtracer_within_reference_noise(fmt):
    """Phong and Blinn-Phong (reflectance 0.5 and 1, exponents 8 and 256) at
    depth 4: per-pixel RMSE against the 4096-spp render within the reference's
    own at equal spp (four reference seeds, render_phong.npz), rays traced
    within the reference's spread."""
    spec, w, h = _phong()
    g = np.load(os.path.join(GOLD, "render_phong.npz"))
    txy, truth = _truth("phong_pt")
    xy = g["pt_xy"]
    assert np.array_equal(xy, txy)
    R = g["pt_rgba"]
    sc = xtgpu.Scene(spec, node_formats=(fmt,))
    frames, rays = [], []
    for seed in (5, 6):
        img, r = sc.render(xtgpu.PATHTRACER, w, h, spp=int(g["spp"]), rdepth=int(g["depth"]), seed=seed,
                           node_format=fmt)
        frames.append(img[xy[:, 1], xy[:, 0]])
        rays.append(r)
    sc.close()
    parity.converged_rmse_bar(np.stack(frames), truth, [parity.rmse(r, truth) for r in R], "phong fmt %d" % fmt)
    ref_rays = g["pt_rays"].astype(np.float64)
    # the GPU scores a lobe without a direction as a miss instead of tracing it
    assert abs(np.mean(rays) - ref_rays.mean()) <= 5 * ref_rays.std() + 0.005 * ref_rays.mean(), (rays, ref_rays)


def test_phong_same_stream_as_oracle():
    """The specular lobe in FP64 on the GPU (sample.inl:61-90, step by step)
    follows the oracle path by path.  The centre pixel's ray meets a Phong
    sphere head-on (identity frame), where most lobe vectors underflow and the
    next ray has no direction: the GPU scores those as the environment in
    that direction, as the reference's ray meets nothing; the centre pixel
    equals the oracle's within 1e-5."""
    spec, w, h = _phong()
    sc = xtgpu.Scene(spec)
    img, rays = sc.render(xtgpu.PATHTRACER, w, h, spp=16, rdepth=4, seed=123)
    sc.close()
    orc = po.OracleScene(spec, po.XO_ACCEL_BVH)
    ys, xs = np.mgrid[0:h, 0:w]
    px = np.stack([xs.ravel(), ys.ravel()], 1)
    o, orays = orc.render(po.PATHTRACER, w, h, spp=16, rdepth=4, seed=123, pixels=px)
    o2, _ = orc.render(po.PATHTRACER, w, h, spp=16, rdepth=4, seed=124, pixels=px)
    parity.same_stream_bar(img, o, o2, "phong pt")
    centre = img[h // 2, w // 2].astype(np.float64)
    oc = o.reshape(h, w, 4)[h // 2, w // 2].astype(np.float64)
    print("[phong centre] gpu %s oracle %s" % (centre, oc))
    assert np.allclose(centre, oc, rtol=1e-5, atol=1e-6)
    assert abs(rays - orays) <= 0.01 * orays


def test_render_is_deterministic_and_rect_consistent():
    spec, w, h = small_scenes()["terrain20k"]
    sc = xtgpu.Scene(spec)
    a, _ = sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=5)
    b, _ = sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=5)
    assert np.array_equal(a, b)
    c, _ = sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=5, rect=(10, 7, 50, 31))
    assert np.array_equal(c, a[7:31, 10:50])
    sc.close()


@pytest.mark.parametrize("integ", [xtgpu.AO, xtgpu.PATHTRACER])
def test_frame_split_into_many_waves_equals_one_wave(integ):
    """A frame rendered in 16 waves of 65,536 paths equals the frame rendered in
    one wave.  The waves are queued back to back without host synchronisation,
    so every wave must keep its own job table until its copies have run."""
    spec, _, _ = small_scenes()["terrain20k"]
    sc = xtgpu.Scene(spec)
    keep = xtgpu.get_tuning().wave_paths
    try:
        xtgpu.set_tuning(wave_paths=1 << 22)
        one, r1 = sc.render(integ, 256, 256, spp=16, rdepth=4, ao_max_distance=0.5, seed=3)
        xtgpu.set_tuning(wave_paths=1 << 16)
        many, r2 = sc.render(integ, 256, 256, spp=16, rdepth=4, ao_max_distance=0.5, seed=3)
    finally:
        xtgpu.set_tuning(wave_paths=keep)
    sc.close()
    assert r1 == r2
    assert np.array_equal(one, many)


def test_bad_arguments_return_invalid():
    spec, w, h = small_scenes()["spheres64"]
    sc = xtgpu.Scene(spec)
    with pytest.raises(xtgpu.XtgpuError) as e:
        sc.render(xtgpu.STENCIL, 0, 10)
    assert e.value.status == 1
    with pytest.raises(xtgpu.XtgpuError) as e:
        sc.render(xtgpu.AO, 8, 8, ao_max_distance=0.0)
    assert e.value.status == 1
    with pytest.raises(xtgpu.XtgpuError) as e:
        sc.render(xtgpu.STENCIL, 8, 8, node_format=xtgpu.NODES_Q8)   # not built
    assert e.value.status == 7
    sc.close()


def _primary_scene(name):
    return {"spheres64": lambda: scenes.spheres_scene(64, seed=1, name="spheres64"),
            "terrain20k": lambda: scenes.terrain_scene(20_000, seed=2, name="terrain20k"),
            "uvscene": lambda: scenes.uv_scene(6)}[name]()


@pytest.mark.parametrize("name", ["spheres64", "terrain20k", "uvscene"])
@pytest.mark.parametrize("integ,code", [("normal", xtgpu.NORMAL), ("uv", xtgpu.UV), ("emission", xtgpu.EMISSION),
                                        ("wireframe", xtgpu.WIREFRAME)])
@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
def test_primary_integrators_vs_reference_golden(name, integ, code, fmt):
    """normal, uv, emission and wireframe frames against the reference's own
    renders (3 samples per pixel, so the per-sample folds are exercised).
    Wireframe and emission fold the same floats as the reference; normal and
    uv carry the FP32 hit point into their FP64 arithmetic (1e-4)."""
    g = np.load(os.path.join(GOLD, "render_primary_%s.npz" % name))
    spec = _primary_scene(name)
    w, h, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    sc = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    img, rays = sc.render(code, w, h, spp=spp, node_format=fmt)
    sc.close()
    assert rays == int(g["%s_rays" % integ]) == w * h * spp
    xy = g["%s_xy" % integ]
    got = img[xy[:, 1], xy[:, 0]]
    ref = g["%s_rgba" % integ]
    nan_g, nan_r = np.isnan(got).any(axis=1), np.isnan(ref).any(axis=1)
    assert np.mean(nan_g == nan_r) >= 0.999
    both = ~nan_g & ~nan_r
    d = np.abs(got[both] - ref[both]).max(axis=1)
    if integ in ("emission", "wireframe"):
        assert np.mean(d == 0) >= 0.999, np.sort(d)[-5:]
    else:
        assert np.mean(d <= 1e-4) >= 0.995, np.sort(d)[-5:]
