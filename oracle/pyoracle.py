"""ctypes binding of the oracle restatement (oracle/xtoracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker.  The product library never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libxtoracle.so")
REF_BIN = os.path.join(HERE, "_ref", "xtref")

XO_ACCEL_OCTREE, XO_ACCEL_BVH = 0, 1
STENCIL, DEPTH, AO, PATHTRACER, NORMAL, UV, EMISSION, WIREFRAME = 0, 1, 2, 3, 4, 5, 6, 7
INTEGRATOR_NAMES = {STENCIL: "stencil", DEPTH: "depth", AO: "ao", PATHTRACER: "pathtracer"}


class XoMaterial(C.Structure):
    _fields_ = [("type", C.c_int32), ("diffuse", C.c_float * 3), ("specular", C.c_float * 3),
                ("emissive", C.c_float * 3), ("reflectance", C.c_float), ("exponent", C.c_float),
                ("ior", C.c_float)]


class XoTexture(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("filtering", C.c_int32), ("pad", C.c_int32),
                ("offset", C.c_int64)]


class XoSampler(C.Structure):
    _fields_ = [("kind", C.c_int32), ("texture", C.c_int32), ("a", C.c_float * 3), ("b", C.c_float * 3)]


def texture_structs(textures, struct=None):
    """(K, 4) rows (width, height, filtering, first texel) as a ctypes array."""
    struct = struct or XoTexture
    out = (struct * max(1, len(textures)))()
    for i, (w, h, f, off) in enumerate(np.asarray(textures).tolist()):
        out[i].width, out[i].height, out[i].filtering, out[i].offset = int(w), int(h), int(f), int(off)
    return out


def sampler_structs(samp, struct=None):
    """Per material three (kind, texture, a, b) tuples as a ctypes array."""
    struct = struct or XoSampler
    out = (struct * max(1, 3 * len(samp)))()
    for i, row in enumerate(samp):
        for ch, (kind, tex, a, b) in enumerate(row):
            k = out[3 * i + ch]
            k.kind, k.texture = int(kind), int(tex)
            k.a[:] = [float(v) for v in a]
            k.b[:] = [float(v) for v in b]
    return out


class XoSceneDesc(C.Structure):
    _fields_ = [("n_objects", C.c_int32), ("obj_kind", C.c_void_p), ("obj_first", C.c_void_p),
                ("obj_count", C.c_void_p), ("obj_material", C.c_void_p),
                ("n_spheres", C.c_int32), ("spheres", C.c_void_p),
                ("n_planes", C.c_int32), ("planes", C.c_void_p),
                ("n_tris", C.c_int32), ("tris", C.c_void_p), ("tri_normals", C.c_void_p),
                ("n_materials", C.c_int32), ("materials", C.c_void_p),
                ("env_type", C.c_int32), ("env_a", C.c_float * 3), ("env_b", C.c_float * 3),
                ("cam_pos", C.c_float * 3), ("cam_target", C.c_float * 3), ("cam_up", C.c_float * 3),
                ("cam_fov", C.c_float), ("obj_uv_scale", C.c_void_p), ("tri_uvs", C.c_void_p),
                ("cam_type", C.c_int32), ("cam_orientation", C.c_float * 3), ("cam_ipd", C.c_float),
                ("cam_flength", C.c_float), ("cam_aperture", C.c_float),
                ("n_textures", C.c_int32), ("textures", C.c_void_p), ("texels", C.c_void_p),
                ("mat_samplers", C.c_void_p), ("env_texture", C.c_int32)]


SAMPLES_GRID, SAMPLES_RANDOM = 0, 1   # aa.h SAMPLE_DISTRIBUTION


def sample_positions(aa: int, distribution: int = SAMPLES_GRID) -> int:
    """Positions per pixel: aa^2 on the grid (aa.cc:7-32), aa jittered ones
    (aa.cc:34-48); level 0 renders as level 1."""
    L = max(int(aa), 1)
    return L if distribution == SAMPLES_RANDOM else L * L


class XoRenderParams(C.Structure):
    _fields_ = [("integrator", C.c_int32), ("width", C.c_int32), ("height", C.c_int32),
                ("spp", C.c_int32), ("rdepth", C.c_int32), ("aa", C.c_int32), ("ao_max_distance", C.c_float),
                ("seed", C.c_uint64), ("distribution", C.c_int32)]


_lib = None


def build() -> None:
    subprocess.run(["sh", os.path.join(HERE, "build_oracle.sh")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.xo_scene_create.argtypes = [C.POINTER(XoSceneDesc), C.c_int, C.POINTER(C.c_void_p)]
        L.xo_scene_destroy.argtypes = [C.c_void_p]
        L.xo_trace.argtypes = [C.c_void_p, C.c_int64] + [C.c_void_p] * 8
        L.xo_camera_ray.argtypes = [C.c_void_p] * 3 + [C.c_float] * 5 + [C.c_void_p] * 2
        L.xo_render_raygraph.argtypes = [C.c_void_p, C.POINTER(XoRenderParams), C.c_int64, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]
        L.xo_render.argtypes = [C.c_void_p, C.POINTER(XoRenderParams), C.c_int64, C.c_void_p,
                                C.c_void_p, C.POINTER(C.c_uint64)]
        for n in ("xo_kat_sphere", "xo_kat_plane"):
            getattr(L, n).argtypes = [C.c_void_p] * 4
        L.xo_kat_triangle.argtypes = [C.c_void_p] * 5
        L.xo_kat_aabb.argtypes = [C.c_void_p] * 4
        L.xo_kat_hemisphere.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.xo_kat_diffuse.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.xo_kat_lobe.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        L.xo_kat_material.argtypes = [C.POINTER(XoMaterial), C.c_void_p, C.c_int32] + [C.c_void_p] * 4
        L.xo_kat_gradient.argtypes = [C.c_void_p] * 4
        L.xo_kat_texture.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p]
        L.xo_kat_erp.argtypes = [C.c_void_p] * 4
        L.xo_kat_cubemap.argtypes = [C.c_void_p] * 4
        L.xo_kat_camera_dof.argtypes = [C.c_void_p, C.c_int32] + [C.c_void_p] * 3 + [C.c_float] * 7 + [C.c_void_p] * 2
        L.xo_kat_camera_erp.argtypes = [C.c_void_p] * 2 + [C.c_float] * 4 + [C.c_void_p] * 2
        L.xo_kat_camera_ods.argtypes = [C.c_void_p] * 2 + [C.c_float] * 5 + [C.c_void_p] * 2
        L.xo_kat_camera_cubemap.argtypes = [C.c_void_p] + [C.c_float] * 4 + [C.c_void_p] * 2
        L.xo_stream_uniform.argtypes = [C.c_uint64, C.c_uint32]
        L.xo_stream_uniform.restype = C.c_double
        L.xo_path_key.argtypes = [C.c_uint64, C.c_uint64]
        L.xo_path_key.restype = C.c_uint64
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleScene:
    """The restated reference scene (Scene + ISurface objects + Octree/BVH)."""

    def __init__(self, spec, accel: int = XO_ACCEL_BVH):
        self.spec = spec
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        d = XoSceneDesc()
        d.n_objects = len(spec.obj_kind)
        d.obj_kind = _ptr(arr(spec.obj_kind, np.int32))
        d.obj_first = _ptr(arr(spec.obj_first, np.int32))
        d.obj_count = _ptr(arr(spec.obj_count, np.int32))
        d.obj_material = _ptr(arr(spec.obj_material, np.int32))
        d.n_spheres = spec.spheres.shape[0]
        d.spheres = _ptr(arr(spec.spheres.reshape(-1), np.float32))
        d.n_planes = spec.planes.shape[0]
        d.planes = _ptr(arr(spec.planes.reshape(-1), np.float32))
        d.n_tris = spec.tris.shape[0]
        d.tris = _ptr(arr(spec.tris.reshape(-1), np.float32))
        d.tri_normals = _ptr(arr(spec.tri_normals.reshape(-1), np.float32)) if spec.tri_normals is not None else None
        mats = (XoMaterial * max(1, len(spec.materials)))()
        for i, m in enumerate(spec.materials):
            mats[i].type = m.type
            mats[i].diffuse[:] = list(m.diffuse)
            mats[i].specular[:] = list(m.specular)
            mats[i].emissive[:] = list(m.emissive)
            mats[i].reflectance = m.reflectance
            mats[i].exponent = m.exponent
            mats[i].ior = m.ior
        self._keep.append(mats)
        d.n_materials = len(spec.materials)
        d.materials = C.cast(mats, C.c_void_p)
        d.env_type = spec.env_type
        d.env_a[:] = list(spec.env_a)
        d.env_b[:] = list(spec.env_b)
        d.cam_pos[:] = list(spec.camera.position)
        d.cam_target[:] = list(spec.camera.target)
        d.cam_up[:] = list(spec.camera.up)
        d.cam_fov = spec.camera.fov
        d.cam_type = getattr(spec.camera, "type", 0)
        d.cam_orientation[:] = list(getattr(spec.camera, "orientation", (0.0, 0.0, 0.0)))
        d.cam_ipd = getattr(spec.camera, "ipd", 0.0)
        d.cam_flength = getattr(spec.camera, "flength", 0.0)
        d.cam_aperture = getattr(spec.camera, "aperture", 0.0)
        uvs = getattr(spec, "obj_uv_scale", None)
        d.obj_uv_scale = _ptr(arr(uvs.reshape(-1), np.float32)) if uvs is not None else None
        tuv = getattr(spec, "tri_uvs", None)
        d.tri_uvs = _ptr(arr(tuv.reshape(-1), np.float32)) if tuv is not None else None
        d.env_texture = -1
        if hasattr(spec, "texture_tables"):
            textures, texels, samp, env_tex = spec.texture_tables()
            tstructs, sstructs = texture_structs(textures), sampler_structs(samp)
            self._keep += [tstructs, sstructs]
            d.n_textures = len(textures)
            d.textures = C.cast(tstructs, C.c_void_p)
            d.texels = _ptr(arr(texels.reshape(-1), np.float32))
            d.mat_samplers = C.cast(sstructs, C.c_void_p) if samp else None
            d.env_texture = env_tex
        self._desc = d
        h = C.c_void_p()
        if lib().xo_scene_create(C.byref(d), accel, C.byref(h)) != 0:
            raise RuntimeError("xo_scene_create failed")
        self.handle = h

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                lib().xo_scene_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def trace(self, org: np.ndarray, dirs: np.ndarray):
        org = np.ascontiguousarray(org, np.float64).reshape(-1, 3)
        dirs = np.ascontiguousarray(dirs, np.float64).reshape(-1, 3)
        n = org.shape[0]
        hit = np.zeros(n, np.int32); t = np.zeros(n); obj = np.zeros(n, np.int32); prim = np.zeros(n, np.int32)
        pt = np.zeros((n, 3)); nr = np.zeros((n, 3))
        lib().xo_trace(self.handle, n, _ptr(org), _ptr(dirs), _ptr(hit), _ptr(t), _ptr(obj), _ptr(prim),
                       _ptr(pt), _ptr(nr))
        return dict(hit=hit, t=t, obj=obj, prim=prim, point=pt, normal=nr)

    def render(self, integrator: int, width: int, height: int, spp: int = 1, rdepth: int = 4,
               ao_max_distance: float = 100.0, seed: int = 1, pixels: np.ndarray = None, aa: int = 1,
               distribution: int = SAMPLES_GRID):
        if pixels is None:
            ys, xs = np.mgrid[0:height, 0:width]
            pixels = np.stack([xs.ravel(), ys.ravel()], axis=1)
        pixels = np.ascontiguousarray(pixels, np.int32).reshape(-1, 2)
        p = XoRenderParams(integrator, width, height, spp, rdepth, aa, ao_max_distance, seed, distribution)
        out = np.zeros((pixels.shape[0], 4), np.float32)
        rays = C.c_uint64(0)
        lib().xo_render(self.handle, C.byref(p), pixels.shape[0], _ptr(pixels), _ptr(out), C.byref(rays))
        return out, int(rays.value)


    def render_raygraph(self, width: int, height: int, spp: int = 1, aa: int = 1, pixels: np.ndarray = None,
                        distribution: int = SAMPLES_GRID):
        """The depth integrator's frame and raygraph records (origin, hit point,
        colour after the sample: 10 per sample, pixels in the given order)."""
        pixels = np.ascontiguousarray(pixels, np.int32).reshape(-1, 2)
        p = XoRenderParams(DEPTH, width, height, spp, 1, aa, 100.0, 1, distribution)
        out = np.zeros((pixels.shape[0], 4), np.float32)
        n = pixels.shape[0] * sample_positions(aa, distribution) * spp
        rec = np.zeros((n, 10), np.float64)
        rays = C.c_uint64(0)
        lib().xo_render_raygraph(self.handle, C.byref(p), pixels.shape[0], _ptr(pixels), _ptr(out), _ptr(rec),
                                 C.byref(rays))
        return out, rec


def raygraph_pixel_order(width: int, height: int, tile_size: int = 32) -> np.ndarray:
    """Pixels in the order the reference's raygraph lists their samples: tiles
    of segment_framebuffer (tile.cc:67-94, row by row), and inside a tile the
    order antialiasing::produce queues them (aa.cc:55-58: column by column)."""
    out = []
    for y0 in range(0, height, tile_size):
        for x0 in range(0, width, tile_size):
            for x in range(x0, min(x0 + tile_size, width)):
                for y in range(y0, min(y0 + tile_size, height)):
                    out.append((x, y))
    return np.array(out, np.int32)


def raygraph_ply(records) -> str:
    """raygraph::write (util/raygraph.cc:8-75) of two-sample paths: the origin
    with the default colour (0, 0, 0) and the hit point with the pixel's colour;
    numbers as an ostream prints them (6 significant digits, %g)."""
    rec = np.asarray(records, np.float64).reshape(-1, 10)
    n = rec.shape[0]
    g = lambda v: "%g" % v
    head = ["ply", "format ascii 1.0", "comment object: A single line", "element vertex %d" % (2 * n),
            "property float x", "property float y", "property float z", "property float red",
            "property float green", "property float blue", "element edge %d" % n, "property int vertex1",
            "property int vertex2", "end_header"]
    lines = []
    for r in rec.tolist():
        lines.append("%s %s %s 0 0 0" % (g(r[0]), g(r[1]), g(r[2])))
        lines.append("%s %s %s %s %s %s" % (g(r[3]), g(r[4]), g(r[5]), g(r[6]), g(r[7]), g(r[8])))
    edges = ["%d %d" % (2 * k, 2 * k + 1) for k in range(n)]
    return "\n".join(head + lines + edges) + "\n"


def camera_rays(spec, width: int, height: int, pixels: np.ndarray):
    """Pixel-centre primary rays (x+0.5, y+0.5) in FP64."""
    pixels = np.asarray(pixels).reshape(-1, 2)
    n = pixels.shape[0]
    org = np.zeros((n, 3)); dirs = np.zeros((n, 3))
    cam = spec.camera
    pos = (C.c_float * 3)(*cam.position); tgt = (C.c_float * 3)(*cam.target); up = (C.c_float * 3)(*cam.up)
    o = np.zeros(3); d = np.zeros(3)
    L = lib()
    for i in range(n):
        L.xo_camera_ray(C.cast(pos, C.c_void_p), C.cast(tgt, C.c_void_p), C.cast(up, C.c_void_p), cam.fov,
                        float(pixels[i, 0]) + 0.5, float(pixels[i, 1]) + 0.5, float(width), float(height),
                        _ptr(o), _ptr(d))
        org[i] = o; dirs[i] = d
    return org, dirs


def path_key(seed: int, path: int) -> int:
    return int(lib().xo_path_key(seed, path))


def stream_uniform(key: int, counter: int) -> float:
    return float(lib().xo_stream_uniform(key, counter))


# ----------------------------------------------------------------------
# The reference itself (oracle/_ref/xtref, built from the XTracer sources).
def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def ref_render(scn: str, integrator: str, width: int, height: int, spp: int = 1, aa: int = 1, rdepth: int = 4,
               threads: int = 1, seed: int = 1, tiles=None, ao_max_distance: float = None, workdir: str = "/tmp",
               raygraph: str = None, distribution: int = SAMPLES_GRID):
    """Runs the reference integrator through IIntegrator::render on the given tiles
    ((x0,y0,x1,y1) list, or None for 32-pixel tiles over the frame).  Returns
    (pixels xy, rgba, stats dict with render_s / rays / threads).  raygraph: a
    path to write the tiles' raygraph to as PLY (the GUI's export).  The random
    distribution's offsets come from libc rand(), seeded once from time()."""
    import json
    import tempfile
    fd, out = tempfile.mkstemp(suffix=".bin", dir=workdir)
    os.close(fd)
    tfile = "-"
    if tiles is not None:
        fd, tfile = tempfile.mkstemp(suffix=".txt", dir=workdir)
        with os.fdopen(fd, "w") as fh:
            fh.write("".join("%d %d %d %d\n" % tuple(t) for t in tiles))
    cmd = [REF_BIN, "render", scn, integrator, str(width), str(height), str(spp), str(aa), str(rdepth),
           str(threads), str(seed), tfile, out]
    if ao_max_distance is not None or raygraph or distribution:
        cmd.append(repr(float(ao_max_distance if ao_max_distance is not None else 100.0)))
    if raygraph or distribution:
        cmd.append(raygraph or "-")
    if distribution:
        cmd.append(str(int(distribution)))
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("xtref render failed: %s %s" % (r.stdout, r.stderr))
    stats = json.loads(r.stdout.strip().splitlines()[-1])
    raw = open(out, "rb").read()
    os.unlink(out)
    if tfile != "-":
        os.unlink(tfile)
    n = int(np.frombuffer(raw[:8], np.int64)[0])
    rec = np.frombuffer(raw[8:], dtype=np.dtype([("xy", np.int32, 2), ("rgba", np.float32, 4)]), count=n)
    return rec["xy"].copy(), rec["rgba"].copy(), stats


def ref_bench(scn: str, integrator: str, width: int, height: int, spp: int, rdepth: int, threads: int, seed: int,
              tiles, repeats: int, workdir: str = "/tmp"):
    """The reference renderer as the timed CPU baseline: loads the scene once
    (load and octree build timed on their own), then runs
    IIntegrator::render `repeats` times over the same tiles.  Returns
    {"load_s", "threads", "renders": [{"render_s", "rays"}, ...]}."""
    import json
    import tempfile
    fd, tfile = tempfile.mkstemp(suffix=".txt", dir=workdir)
    with os.fdopen(fd, "w") as fh:
        fh.write("".join("%d %d %d %d\n" % tuple(t) for t in tiles))
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    cmd = [REF_BIN, "bench", scn, integrator, str(width), str(height), str(spp), str(rdepth), str(threads),
           str(seed), tfile, str(repeats)]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    os.unlink(tfile)
    if r.returncode != 0:
        raise RuntimeError("xtref bench failed: %s %s" % (r.stdout, r.stderr))
    return json.loads(r.stdout.strip().splitlines()[-1])


def ref_hits(scn: str, width: int, height: int, tiles=None, obj_path: str = None, workdir: str = "/tmp"):
    """Primary-ray closest hits through the reference's Scene::intersection, plus
    the triangle index from an Octree<Triangle> replica of the mesh."""
    import tempfile
    fd, out = tempfile.mkstemp(suffix=".bin", dir=workdir)
    os.close(fd)
    tfile = "-"
    if tiles is not None:
        fd, tfile = tempfile.mkstemp(suffix=".txt", dir=workdir)
        with os.fdopen(fd, "w") as fh:
            fh.write("".join("%d %d %d %d\n" % tuple(t) for t in tiles))
    cmd = [REF_BIN, "hits", scn, str(width), str(height), tfile, out] + ([obj_path] if obj_path else [])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("xtref hits failed: %s %s" % (r.stdout, r.stderr))
    raw = open(out, "rb").read()
    os.unlink(out)
    if tfile != "-":
        os.unlink(tfile)
    n = int(np.frombuffer(raw[:8], np.int64)[0])
    nobj = int(np.frombuffer(raw[8:12], np.int32)[0])
    names = [raw[12 + 64 * i:12 + 64 * (i + 1)].split(b"\0")[0].decode() for i in range(nobj)]
    off = 12 + 64 * nobj
    dt = np.dtype([("xy", np.int32, 2), ("hi", np.int32, 3), ("rec", np.float64, 14)])
    rec = np.frombuffer(raw[off:], dtype=dt, count=n)
    r = rec["rec"]
    return dict(xy=rec["xy"].copy(), hit=rec["hi"][:, 0].copy(), obj=rec["hi"][:, 1].copy(),
                prim=rec["hi"][:, 2].copy(), org=r[:, 0:3].copy(), dir=r[:, 3:6].copy(), t=r[:, 6].copy(),
                point=r[:, 7:10].copy(), normal=r[:, 10:13].copy(), t_replica=r[:, 13].copy(), names=names)


def ref_kat(lines, workdir: str = "/tmp"):
    """Runs known-answer lines ("kind a b c ...", numbers as hex floats) through
    the reference functions; returns the output lines split into tokens."""
    import tempfile
    fd, fin = tempfile.mkstemp(suffix=".txt", dir=workdir)
    with os.fdopen(fd, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    fd, fout = tempfile.mkstemp(suffix=".txt", dir=workdir)
    os.close(fd)
    r = subprocess.run([REF_BIN, "kat", fin, fout], capture_output=True, text=True)
    os.unlink(fin)
    if r.returncode != 0:
        raise RuntimeError("xtref kat failed: %s" % r.stderr)
    res = [ln.split() for ln in open(fout).read().splitlines()]
    os.unlink(fout)
    return res
