"""ctypes binding of libxtgpu.so (include/xtgpu.h) and a thin Python mirror of
XTracer's renderer interface for the hot path:

* ``Scene``            a flattened, resident xtcore Scene (scene.h:35-86) with its
                       LBVH; ``Scene.intersection`` is Scene::intersection
                       (scene.cc:191-216) over a batch of rays.
* ``Params``           params_t (context.h:18-34): width, height, samples, rdepth.
* ``StencilIntegrator``, ``DepthIntegrator``, ``AOIntegrator``,
  ``PathtracerIntegrator``: IIntegrator (integrator.h:10-24) with setup() and
  render(); render() returns the RGBA frame the reference assembles from its
  tiles (context.cc:38-52).

The CUDA library is required: nothing here falls back to a CPU path.  Errors
raise XtgpuError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libxtgpu.so")

STENCIL, DEPTH, AO, PATHTRACER, NORMAL, UV, EMISSION, WIREFRAME = 0, 1, 2, 3, 4, 5, 6, 7
NODES_FP32, NODES_Q8, NODES_W8 = 0, 1, 2
# bytes one node visit reads, per format
NODE_BYTES = {NODES_FP32: 64, NODES_Q8: 32, NODES_W8: 80}
STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "LIMIT", 5: "TIMEOUT", 6: "NOT_FOUND", 7: "STATE"}


class XtgpuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("diffuse", C.c_float * 3), ("specular", C.c_float * 3),
                ("emissive", C.c_float * 3), ("reflectance", C.c_float), ("exponent", C.c_float),
                ("ior", C.c_float)]


class CameraDesc(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3), ("fov", C.c_float),
                ("type", C.c_int32), ("orientation", C.c_float * 3), ("ipd", C.c_float), ("flength", C.c_float),
                ("aperture", C.c_float)]


class Texture(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("filtering", C.c_int32), ("reserved", C.c_int32),
                ("offset", C.c_int64)]


class SamplerDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("texture", C.c_int32), ("a", C.c_float * 3), ("b", C.c_float * 3)]


class SceneDesc(C.Structure):
    _fields_ = [("n_objects", C.c_int32), ("obj_kind", C.c_void_p), ("obj_first", C.c_void_p),
                ("obj_count", C.c_void_p), ("obj_material", C.c_void_p),
                ("n_spheres", C.c_int32), ("spheres", C.c_void_p),
                ("n_planes", C.c_int32), ("planes", C.c_void_p),
                ("n_tris", C.c_int32), ("tris", C.c_void_p), ("tri_normals", C.c_void_p),
                ("n_materials", C.c_int32), ("materials", C.c_void_p),
                ("env_type", C.c_int32), ("env_a", C.c_float * 3), ("env_b", C.c_float * 3),
                ("camera", CameraDesc), ("obj_uv_scale", C.c_void_p), ("tri_uvs", C.c_void_p),
                ("n_textures", C.c_int32), ("textures", C.c_void_p), ("n_texels", C.c_int64),
                ("texels", C.c_void_p), ("mat_samplers", C.c_void_p), ("env_texture", C.c_int32)]


class BvhOpts(C.Structure):
    _fields_ = [("node_format", C.c_int32), ("leaf_size", C.c_int32)]


class BvhInfo(C.Structure):
    _fields_ = [("n_prims", C.c_int64), ("depth", C.c_int32), ("leaf_size", C.c_int32),
                ("node_bytes_fp32", C.c_uint64), ("node_bytes_q8", C.c_uint64), ("node_bytes_w8", C.c_uint64),
                ("depth_w8", C.c_int32)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("prim", C.c_uint32), ("u", C.c_float), ("v", C.c_float)]


HIT_DTYPE = np.dtype([("t", np.float32), ("prim", np.uint32), ("u", np.float32), ("v", np.float32)])


# sample distributions (aa.h:14-18)
SAMPLES_GRID, SAMPLES_RANDOM = 0, 1


def sample_positions(aa: int, distribution: int = SAMPLES_GRID) -> int:
    """Positions per pixel: aa^2 on the grid (aa.cc:7-32), aa jittered ones
    (aa.cc:34-48); level 0 renders as level 1."""
    L = max(int(aa), 1)
    return L if distribution == SAMPLES_RANDOM else L * L


class RenderParams(C.Structure):
    _fields_ = [("integrator", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("rdepth", C.c_int32), ("ao_max_distance", C.c_float), ("seed", C.c_uint64),
                ("node_format", C.c_int32), ("x0", C.c_int32), ("y0", C.c_int32), ("x1", C.c_int32),
                ("y1", C.c_int32), ("aa", C.c_int32), ("sample_distribution", C.c_int32)]


class ServiceOpts(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_uint64), ("max_jobs", C.c_int32), ("wave_paths", C.c_int64),
                ("node_format", C.c_int32), ("use_graphs", C.c_int32), ("merge_jobs", C.c_int32),
                ("host_results", C.c_int32), ("time_kernels", C.c_int32), ("count_visits", C.c_int32),
                ("policy", C.c_int32), ("waves_in_flight", C.c_int32)]


class ServiceStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("waves", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("extend_ms", C.c_double), ("extend_launches", C.c_uint64), ("node_visits", C.c_uint64),
                ("prim_tests", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("extend_variant", C.c_int32), ("extend_block", C.c_int32), ("extend_blocks_per_sm", C.c_int32),
                ("tile", C.c_int32), ("wave_paths", C.c_int64), ("leaf_size", C.c_int32),
                ("node_layout", C.c_int32), ("refill_threshold", C.c_int32), ("extend_min_blocks", C.c_int32),
                ("stack_entries", C.c_int32), ("steps_per_vote", C.c_int32),
                ("primary_node_format", C.c_int32), ("primary_variant", C.c_int32), ("bvh_builder", C.c_int32),
                ("wide_collapse", C.c_int32), ("wide_prim_cost", C.c_float)]


def get_tuning() -> "Tuning":
    t = Tuning()
    check(lib().xtgpu_get_tuning(C.byref(t)))
    return t


def set_tuning(**kw) -> None:
    t = get_tuning()
    for k, v in kw.items():
        setattr(t, k, v)
    check(lib().xtgpu_set_tuning(C.byref(t)))


class JobDesc(C.Structure):
    _fields_ = [("scene", C.c_int32), ("integrator", C.c_int32), ("width", C.c_int32), ("height", C.c_int32),
                ("spp", C.c_int32), ("rdepth", C.c_int32), ("ao_max_distance", C.c_float), ("seed", C.c_uint64),
                ("aa", C.c_int32), ("sample_distribution", C.c_int32)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("rays", C.c_uint64), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("finish_s", C.c_double), ("render_done_s", C.c_double)]


# Every entry point of include/xtgpu.h with its argument types.
SIGNATURES = {
    "xtgpu_scene_create": [C.POINTER(SceneDesc), C.c_void_p, C.POINTER(C.c_void_p)],
    "xtgpu_bvh_build": [C.c_void_p, C.POINTER(BvhOpts), C.c_void_p],
    "xtgpu_scene_destroy": [C.c_void_p],
    "xtgpu_scene_device_bytes": [C.c_void_p, C.POINTER(C.c_uint64)],
    "xtgpu_bvh_export": [C.c_void_p, C.POINTER(BvhInfo), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "xtgpu_trace": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p],
    "xtgpu_trace_host": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p],
    "xtgpu_trace_counts": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                           C.c_void_p],
    "xtgpu_render": [C.c_void_p, C.POINTER(RenderParams), C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p],
    "xtgpu_render_host": [C.c_void_p, C.POINTER(RenderParams), C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p],
    "xtgpu_render_tile_noalloc": [C.c_void_p, C.POINTER(RenderParams), C.c_void_p, C.POINTER(C.c_uint64),
                                  C.c_void_p],
    "xtgpu_service_create": [C.POINTER(ServiceOpts), C.c_void_p, C.POINTER(C.c_void_p)],
    "xtgpu_service_add_scene": [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)],
    "xtgpu_service_submit": [C.c_void_p, C.POINTER(JobDesc), C.c_double, C.POINTER(C.c_int64)],
    "xtgpu_service_run": [C.c_void_p, C.c_double],
    "xtgpu_service_open": [C.c_void_p, C.c_int32],
    "xtgpu_service_poll": [C.c_void_p, C.c_int64, C.POINTER(JobStatus)],
    "xtgpu_service_result": [C.c_void_p, C.c_int64, C.c_void_p],
    "xtgpu_service_result_host": [C.c_void_p, C.c_int64, C.POINTER(C.POINTER(C.c_float))],
    "xtgpu_service_release": [C.c_void_p, C.c_int64],
    "xtgpu_service_destroy": [C.c_void_p],
    "xtgpu_service_get_stats": [C.c_void_p, C.POINTER(ServiceStats)],
    "xtgpu_service_reset_stats": [C.c_void_p],
    "xtgpu_get_tuning": [C.c_void_p],
    "xtgpu_set_tuning": [C.c_void_p],
    "xtgpu_autotune": [C.c_void_p, C.c_int32, C.c_double, C.c_void_p, C.c_void_p],
    "xtgpu_scene_tuning": [C.c_void_p, C.c_void_p],
    "xtgpu_scene_set_tuning": [C.c_void_p, C.c_void_p],
    "xtgpu_frame_rgba8": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p],
    "xtgpu_write_png": [C.c_char_p, C.c_int32, C.c_int32, C.c_void_p],
    "xtgpu_write_exr": [C.c_char_p, C.c_int32, C.c_int32, C.c_void_p],
    "xtgpu_save_png_host": [C.c_char_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p],
    "xtgpu_render_raygraph": [C.c_void_p, C.POINTER(RenderParams), C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64),
                              C.c_void_p],
    "xtgpu_render_raygraph_host": [C.c_void_p, C.POINTER(RenderParams), C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_uint64), C.c_void_p],
    "xtgpu_write_raygraph_ply": [C.c_char_p, C.c_int64, C.c_void_p],
    "xtgpu_scene_update": [C.c_void_p, C.POINTER(SceneDesc), C.c_int32, C.c_void_p],
    "xtgpu_service_update_scene": [C.c_void_p, C.c_int32],
}

_lib = None


def lib():
    """Loads libxtgpu.so (building it first if it is missing).  Raises if it
    cannot be built or loaded: there is no CPU fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.xtgpu_last_error.restype = C.c_char_p
        L.xtgpu_version.restype = C.c_char_p
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise XtgpuError(status, lib().xtgpu_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def stream_handle(stream=None) -> Optional[int]:
    """cudaStream_t of a torch.cuda.Stream (or None for the default stream)."""
    if stream is None:
        return None
    return int(getattr(stream, "cuda_stream", stream))


def scene_desc(spec):
    """The C ABI's xtgpu_scene_desc of a scene spec (scenes.SceneSpec), and the
    arrays it points into (keep them alive while the description is used)."""
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return _ptr(a)

    d = SceneDesc()
    d.n_objects = len(spec.obj_kind)
    d.obj_kind = arr(spec.obj_kind, np.int32)
    d.obj_first = arr(spec.obj_first, np.int32)
    d.obj_count = arr(spec.obj_count, np.int32)
    d.obj_material = arr(spec.obj_material, np.int32)
    d.n_spheres = spec.spheres.shape[0]
    d.spheres = arr(spec.spheres.reshape(-1), np.float32)
    d.n_planes = spec.planes.shape[0]
    d.planes = arr(spec.planes.reshape(-1), np.float32)
    d.n_tris = spec.tris.shape[0]
    d.tris = arr(spec.tris.reshape(-1), np.float32)
    d.tri_normals = arr(spec.tri_normals.reshape(-1), np.float32) if spec.tri_normals is not None else None
    mats = (Material * max(1, len(spec.materials)))()
    for i, m in enumerate(spec.materials):
        mats[i].type = m.type
        mats[i].diffuse[:] = list(m.diffuse)
        mats[i].specular[:] = list(m.specular)
        mats[i].emissive[:] = list(m.emissive)
        mats[i].reflectance, mats[i].exponent, mats[i].ior = m.reflectance, m.exponent, m.ior
    keep.append(mats)
    d.n_materials = len(spec.materials)
    d.materials = C.cast(mats, C.c_void_p)
    d.env_type = spec.env_type
    d.env_a[:] = list(spec.env_a)
    d.env_b[:] = list(spec.env_b)
    cam = spec.camera
    d.camera.position[:] = list(cam.position)
    d.camera.target[:] = list(cam.target)
    d.camera.up[:] = list(cam.up)
    d.camera.fov = cam.fov
    d.camera.type = getattr(cam, "type", 0)
    d.camera.orientation[:] = list(getattr(cam, "orientation", (0.0, 0.0, 0.0)))
    d.camera.ipd = getattr(cam, "ipd", 0.0)
    d.camera.flength = getattr(cam, "flength", 0.0)
    d.camera.aperture = getattr(cam, "aperture", 0.0)
    if getattr(spec, "obj_uv_scale", None) is not None:
        d.obj_uv_scale = arr(spec.obj_uv_scale.reshape(-1), np.float32)
    if getattr(spec, "tri_uvs", None) is not None:
        d.tri_uvs = arr(spec.tri_uvs.reshape(-1), np.float32)
    d.env_texture = -1
    if hasattr(spec, "texture_tables"):
        # textures, texels and the materials' samplers (sampler_*.cc)
        textures, texels, samp, env_tex = spec.texture_tables()
        tex = (Texture * max(1, len(textures)))()
        for i, (w, h, f, off) in enumerate(np.asarray(textures).tolist()):
            tex[i].width, tex[i].height, tex[i].filtering, tex[i].offset = int(w), int(h), int(f), int(off)
        sam = (SamplerDesc * max(1, 3 * len(samp)))()
        for i, row in enumerate(samp):
            for ch, (kind, t, a, b) in enumerate(row):
                k = sam[3 * i + ch]
                k.kind, k.texture = int(kind), int(t)
                k.a[:] = [float(v) for v in a]
                k.b[:] = [float(v) for v in b]
        keep += [tex, sam]
        d.n_textures = len(textures)
        d.textures = C.cast(tex, C.c_void_p)
        d.n_texels = int(texels.shape[0])
        d.texels = arr(texels.reshape(-1), np.float32)
        d.mat_samplers = C.cast(sam, C.c_void_p) if samp else None
        d.env_texture = env_tex
    return d, keep


class Scene:
    """A flattened xtcore Scene resident on the current CUDA device."""

    def __init__(self, spec, node_formats=(NODES_FP32,), leaf_size: int = 2, stream=None):
        self.spec = spec
        d, self._keep = scene_desc(spec)
        h = C.c_void_p()
        check(lib().xtgpu_scene_create(C.byref(d), stream_handle(stream), C.byref(h)))
        self.handle = h
        self.formats = set()
        for f in node_formats:
            self.build_bvh(f, leaf_size, stream)

    def update(self, spec, what: int = 3, stream=None) -> None:
        """xtgpu_scene_update from a spec of the same geometry: what = 1
        (UPDATE_SHADING) the materials, samplers, textures, object materials
        and environment, 2 (UPDATE_CAMERA) the camera, 3 both."""
        d, keep = scene_desc(spec)
        check(lib().xtgpu_scene_update(self.handle, C.byref(d), what, stream_handle(stream)))
        self.spec = spec

    def build_bvh(self, node_format: int = NODES_FP32, leaf_size: int = 2, stream=None) -> None:
        o = BvhOpts(node_format, leaf_size)
        check(lib().xtgpu_bvh_build(self.handle, C.byref(o), stream_handle(stream)))
        self.formats.add(node_format)

    def autotune(self, node_format: int = NODES_FP32, budget_ms: float = 3000.0, stream=None) -> "Tuning":
        """Picks this scene's leaf size, stack size, tile, register cap and wave
        size by timing a probe pathtracer job (xtgpu_autotune)."""
        t = Tuning()
        check(lib().xtgpu_autotune(self.handle, node_format, budget_ms, C.byref(t), stream_handle(stream)))
        self.formats.add(node_format)
        return t

    def tuning(self) -> "Tuning":
        t = Tuning()
        check(lib().xtgpu_scene_tuning(self.handle, C.byref(t)))
        return t

    def set_tuning(self, **kw) -> None:
        """Changes fields of the tuning this scene renders with."""
        t = self.tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        check(lib().xtgpu_scene_set_tuning(self.handle, C.byref(t)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().xtgpu_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self) -> int:
        b = C.c_uint64()
        check(lib().xtgpu_scene_device_bytes(self.handle, C.byref(b)))
        return int(b.value)

    def bvh_export(self):
        info = BvhInfo()
        check(lib().xtgpu_bvh_export(self.handle, C.byref(info), None, None, None, None, None))
        n = int(info.n_prims)
        mort = np.zeros(max(n, 1), np.uint32); order = np.zeros(max(n, 1), np.uint32)
        left = np.zeros(max(n - 1, 1), np.int32); right = np.zeros(max(n - 1, 1), np.int32)
        check(lib().xtgpu_bvh_export(self.handle, C.byref(info), _ptr(mort), _ptr(order), _ptr(left), _ptr(right),
                                     None))
        return dict(info=info, morton=mort[:n], order=order[:n], left=left[:max(n - 1, 0)], right=right[:max(n - 1, 0)])

    def intersection(self, org: np.ndarray, dirs: np.ndarray, tmin: float = 0.0, tmax: float = np.inf,
                     node_format: int = NODES_FP32):
        """Closest hits of a batch of rays (host arrays; copies included)."""
        org = np.asarray(org, np.float32).reshape(-1, 3)
        dirs = np.asarray(dirs, np.float32).reshape(-1, 3)
        n = org.shape[0]
        o4 = np.empty((n, 4), np.float32); d4 = np.empty((n, 4), np.float32)
        o4[:, :3] = org; o4[:, 3] = tmin
        d4[:, :3] = dirs; d4[:, 3] = tmax
        hits = np.zeros(n, HIT_DTYPE)
        check(lib().xtgpu_trace_host(self.handle, n, _ptr(o4), _ptr(d4), _ptr(hits), node_format, None))
        return hits

    def render(self, integrator: int, width: int, height: int, spp: int = 1, rdepth: int = 4,
               ao_max_distance: float = 100.0, seed: int = 1, node_format: int = NODES_FP32, rect=None,
               aa: int = 1, distribution: int = SAMPLES_GRID):
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, 0, 0)
        p = RenderParams(integrator, width, height, spp, rdepth, ao_max_distance, seed, node_format, x0, y0, x1, y1,
                         aa, distribution)
        rw, rh = (x1 - x0, y1 - y0) if rect is not None else (width, height)
        out = np.zeros((rh, rw, 4), np.float32)
        rays = C.c_uint64()
        check(lib().xtgpu_render_host(self.handle, C.byref(p), _ptr(out), C.byref(rays), None))
        return out, int(rays.value)

    def render_raygraph(self, width: int, height: int, spp: int = 1, aa: int = 1, node_format: int = NODES_FP32,
                        rect=None, tile_size: int = 32, distribution: int = SAMPLES_GRID):
        """The depth integrator with its raygraph: (frame, records) where the
        records (n, 10: origin, hit point, RGBA after the sample) are listed in
        XTracer's raygraph order (tiles, then columns, then samples)."""
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, 0, 0)
        p = RenderParams(DEPTH, width, height, spp, 1, 100.0, 1, node_format, x0, y0, x1, y1, aa, distribution)
        rw, rh = (x1 - x0, y1 - y0) if rect is not None else (width, height)
        S = sample_positions(aa, distribution) * spp
        out = np.zeros((rh, rw, 4), np.float32)
        rec = np.zeros((rh * rw * S, 10), np.float32)
        rays = C.c_uint64()
        check(lib().xtgpu_render_raygraph_host(self.handle, C.byref(p), _ptr(out), _ptr(rec), C.byref(rays), None))
        px = raygraph_pixel_order(width, height, tile_size, rect if rect is not None else None)
        ox, oy = (x0, y0) if rect is not None else (0, 0)
        pix = (px[:, 1] - oy) * rw + (px[:, 0] - ox)
        order = (pix[:, None] * S + np.arange(S)[None, :]).reshape(-1)
        return out, rec[order]


def raygraph_pixel_order(width: int, height: int, tile_size: int = 32, rect=None) -> np.ndarray:
    """Pixels in the order XTracer's raygraph lists them: the tiles of
    segment_framebuffer (tile.cc:67-94) row by row, and inside a tile column
    by column, as antialiasing::produce queues them (aa.cc:55-58)."""
    x0, y0, x1, y1 = rect if rect is not None else (0, 0, width, height)
    out = []
    for ty in range(0, height, tile_size):
        for tx in range(0, width, tile_size):
            for x in range(max(tx, x0), min(tx + tile_size, width, x1)):
                for y in range(max(ty, y0), min(ty + tile_size, height, y1)):
                    out.append((x, y))
    return np.array(out, np.int32).reshape(-1, 2)


def save_raygraph_ply(path: str, records) -> None:
    """raygraph::write of the records (n, 10), in the order given."""
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 10)
    check(lib().xtgpu_write_raygraph_ply(path.encode(), r.shape[0], _ptr(r)))


class Params:
    """params_t (context.h:18-34) for the GPU integrators."""

    def __init__(self, width=500, height=500, samples=1, rdepth=100, seed=1, node_format=NODES_FP32,
                 ao_max_distance=100.0, aa=1, sample_distribution=SAMPLES_GRID):
        self.width, self.height, self.samples, self.rdepth = width, height, samples, rdepth
        self.seed, self.node_format, self.ao_max_distance = seed, node_format, ao_max_distance
        self.aa, self.sample_distribution = aa, sample_distribution


class Context:
    """context_t (context.h:36-51): a scene plus render parameters."""

    def __init__(self, scene: Scene, params: Params):
        self.scene, self.params = scene, params


class _Integrator:
    kind = None

    def __init__(self):
        self.ctx = None
        self.rays = 0

    def setup(self, context: Context) -> None:   # IIntegrator::setup, integrator.cc:14-17
        self.ctx = context

    def render(self):
        """IIntegrator::render (integrator.cc:29-53) for the whole frame.  Like
        the reference it does nothing without a context."""
        if self.ctx is None:
            return None
        p = self.ctx.params
        img, self.rays = self.ctx.scene.render(self.kind, p.width, p.height, p.samples, p.rdepth,
                                               p.ao_max_distance, p.seed, p.node_format, aa=p.aa,
                                               distribution=p.sample_distribution)
        return img


class StencilIntegrator(_Integrator):
    kind = STENCIL


class DepthIntegrator(_Integrator):
    kind = DEPTH


class AOIntegrator(_Integrator):
    kind = AO


class PathtracerIntegrator(_Integrator):
    kind = PATHTRACER


class NormalIntegrator(_Integrator):
    kind = NORMAL


class UVIntegrator(_Integrator):
    kind = UV


class EmissionIntegrator(_Integrator):
    kind = EMISSION


class WireframeIntegrator(_Integrator):
    kind = WIREFRAME


def save_png(path: str, frame, stream=None) -> None:
    """Writes an RGBA float frame (H, W, 4) as an 8-bit PNG with XTracer's
    quantisation (lib/nimg/img.cc:150-172), done on the GPU: a CUDA tensor is
    quantised in place on its device, a host array is uploaded first."""
    if hasattr(frame, "is_cuda") and frame.is_cuda:
        import torch
        f = frame.contiguous()
        h, w = int(f.shape[0]), int(f.shape[1])
        q = torch.empty((h, w, 4), dtype=torch.uint8, device=f.device)
        check(lib().xtgpu_frame_rgba8(C.c_void_p(f.data_ptr()), h * w, C.c_void_p(q.data_ptr()),
                                      stream_handle(stream)))
        host = q.cpu().numpy()
        check(lib().xtgpu_write_png(path.encode(), w, h, _ptr(np.ascontiguousarray(host))))
        return
    a = np.ascontiguousarray(frame, np.float32)
    check(lib().xtgpu_save_png_host(path.encode(), a.shape[1], a.shape[0], _ptr(a), stream_handle(stream)))


def save_exr(path: str, frame) -> None:
    """Writes the R, G, B channels of an RGBA float frame (H, W, 4) as an
    uncompressed OpenEXR file, the layout XTracer's EXR writer uses
    (lib/nimg/img.cc:72-141)."""
    if hasattr(frame, "is_cuda") and frame.is_cuda:
        frame = frame.cpu().numpy()
    a = np.ascontiguousarray(frame, np.float32)
    check(lib().xtgpu_write_exr(path.encode(), a.shape[1], a.shape[0], _ptr(a)))
