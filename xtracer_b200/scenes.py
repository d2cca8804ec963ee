"""Seeded synthetic scenes and job streams for the ray-intersection hot path.

Every scene is produced from a seed and held as flat float32 arrays (the layout
the C ABI takes, include/xtgpu.h).  The same scene can be written as an XTracer
``.scn`` file (+ ``.obj`` for meshes) so the reference renderer loads exactly the
same numbers:

* all coordinates are rounded to dyadic grids (2^-16 for |x| < 128, 2^-22 inside
  the unit ball), so each value is an exact float32 whose shortest decimal form
  parses back to the same float in the reference's ``sscanf("%f")`` /
  ``strtod`` / tinyobj readers;
* object names are zero-padded (``o00000``...), so the reference's std::map
  iteration order (src/xtcore/scene.cc:191-216) is the order used here.

No public dataset is used; the reference's own sample meshes (scene/data/) are
absent from its repository anyway.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional

import numpy as np

SPHERE, PLANE, MESH = 0, 1, 2
LAMBERT, PHONG, BLINNPHONG, EMISSIVE, DIELECTRIC = 0, 1, 2, 3, 4
ENV_NONE, ENV_COLOR, ENV_GRADIENT, ENV_ERP, ENV_CUBEMAP = 0, 1, 2, 3, 4
MATERIAL_NAMES = {LAMBERT: "lambert", PHONG: "phong", BLINNPHONG: "blinn_phong",
                  EMISSIVE: "emissive", DIELECTRIC: "dielectric"}
# material samplers (sampler_col.cc, sampler_gradient.cc, sampler_tex.cc,
# sampler_erp.cc, sampler_cubemap.cc) and texture filtering (sampler.h:11-15)
SAMPLER_COLOR, SAMPLER_GRADIENT, SAMPLER_TEXTURE, SAMPLER_ERP, SAMPLER_CUBEMAP = 0, 1, 2, 3, 4
FILTER_NEAREST, FILTER_BILINEAR = 0, 1
# the .scn keys of the six cubemap faces in CUBEMAP_FACE order (left, right,
# top, bottom, front, back: sampler_cubemap.h:11-19, parseutil.cc:177-182)
CUBE_FACE_KEYS = ("negx", "posx", "posy", "negy", "posz", "negz")


@dataclasses.dataclass(eq=False)
class Texture:
    """An 8-bit RGB or RGBA image, written as PNG for the reference, which
    loads it with stbi_load and divides each channel by 255.f (alpha 1 for
    RGB, nimg/img.cc:17-66), then applies flip_x / flip_y (sampler_tex.cc)."""
    pixels: np.ndarray                 # (H, W, 3 or 4) uint8, top row first
    filtering: int = FILTER_NEAREST
    flip_x: bool = False
    flip_y: bool = False

    def texels(self) -> np.ndarray:
        """(H, W, 4) float32 as Texture2D holds them after loading."""
        p = np.asarray(self.pixels, np.uint8)
        rgba = np.ones(p.shape[:2] + (4,), np.float32)
        rgba[..., :p.shape[2]] = p.astype(np.float32) / np.float32(255.0)
        if self.flip_x:
            rgba = rgba[:, ::-1]
        if self.flip_y:
            rgba = rgba[::-1]
        return np.ascontiguousarray(rgba)


@dataclasses.dataclass
class Sampler:
    """A material or environment sampler: a colour, a gradient over the
    normalised texcoord (or direction), a 2D texture, an equirectangular map
    or a cubemap (six textures in CUBEMAP_FACE order)."""
    kind: int = SAMPLER_COLOR
    a: tuple = (0.0, 0.0, 0.0)
    b: tuple = (0.0, 0.0, 0.0)
    textures: tuple = ()


@dataclasses.dataclass
class Material:
    type: int = LAMBERT
    diffuse: tuple = (0.0, 0.0, 0.0)
    specular: tuple = (0.0, 0.0, 0.0)
    emissive: tuple = (0.0, 0.0, 0.0)
    reflectance: float = 0.0
    exponent: float = 0.0
    ior: float = 1.0
    # "diffuse" / "specular" / "emissive" -> Sampler, replacing that colour
    samplers: Optional[dict] = None

    def sampler(self, key: str) -> "Sampler":
        if self.samplers and key in self.samplers:
            return self.samplers[key]
        return Sampler(SAMPLER_COLOR, tuple(getattr(self, key)))


def write_png(path: str, pixels: np.ndarray) -> None:
    """8-bit RGB or RGBA PNG (one IDAT, filter 0 on every row)."""
    import struct
    import zlib
    p = np.ascontiguousarray(np.asarray(pixels, np.uint8))
    h, w, c = p.shape
    raw = b"".join(b"\x00" + p[y].tobytes() for y in range(h))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as fh:
        fh.write(b"\x89PNG\r\n\x1a\n")
        fh.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2 if c == 3 else 6, 0, 0, 0)))
        fh.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        fh.write(chunk(b"IEND", b""))


CAM_PERSPECTIVE, CAM_ERP, CAM_ODS, CAM_CUBEMAP = 0, 1, 2, 3
CAMERA_NAMES = {CAM_PERSPECTIVE: "thin-lens", CAM_ERP: "erp", CAM_ODS: "ods", CAM_CUBEMAP: "cubemap"}


@dataclasses.dataclass
class Camera:
    position: tuple = (0.0, 0.0, -10.0)
    target: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    fov: float = 60.0
    type: int = CAM_PERSPECTIVE
    orientation: tuple = (0.0, 0.0, 0.0)   # ERP, ODS: euler angles (radians)
    ipd: float = 0.0                       # ODS: eye separation
    flength: float = 0.0                   # perspective: focal length (depth of field when > 0)
    aperture: float = 0.0


@dataclasses.dataclass
class SceneSpec:
    """Flat scene: objects in intersection order, each a sphere, a plane or a
    mesh (a contiguous range of triangles)."""
    name: str
    spheres: np.ndarray            # (S, 4) float32: cx cy cz r
    planes: np.ndarray             # (P, 4) float32: nx ny nz offset
    tris: np.ndarray               # (T, 3, 3) float32, OBJ face order per mesh
    obj_kind: np.ndarray           # (O,) int32
    obj_first: np.ndarray          # (O,) int32
    obj_count: np.ndarray          # (O,) int32
    obj_material: np.ndarray       # (O,) int32
    materials: List[Material]
    camera: Camera
    env_type: int = ENV_NONE
    env_a: tuple = (0.0, 0.0, 0.0)
    env_b: tuple = (0.0, 0.0, 0.0)
    tri_normals: Optional[np.ndarray] = None
    # mesh vertex/index form for writing OBJ (per mesh object): list of (verts, faces)
    mesh_obj: Optional[list] = None
    # per object (u_scale, v_scale) of the geometry (ISurface::uv_scale; the
    # loader's default is (0, 0)), and per triangle the texcoords of its three
    # corners (Triangle::tc, OBJ "vt"); None = all zero
    obj_uv_scale: Optional[np.ndarray] = None      # (O, 2) float32
    tri_uvs: Optional[np.ndarray] = None           # (T, 3, 2) float32
    # ENV_ERP: one texture; ENV_CUBEMAP: six in CUBEMAP_FACE order
    env_textures: tuple = ()
    # further cameras of the .scn, by name (the scene's own is "default")
    extra_cameras: Optional[dict] = None
    # write every mesh object into one OBJ with an MTL material library, read
    # by the loader's external-object path (parseutil.cc:588-682); the meshes
    # must be the last objects and their materials expressible in MTL
    mtl_meshes: bool = False

    def texture_tables(self):
        """The scene's textures and samplers as the C ABI takes them:
        textures (K, 4) int64 rows (width, height, filtering, first texel),
        texels (N, 4) float32, mat_samplers (M, 3) of (kind, first texture,
        a, b) per diffuse/specular/emissive, env_texture.  A texture object
        used several times is stored once; cubemap faces are consecutive."""
        rows, blocks, index = [], [], {}
        total = 0

        def add(texs):
            nonlocal total
            key = tuple(id(t) for t in texs)
            if key in index:
                return index[key]
            first = len(rows)
            for t in texs:
                tx = t.texels()
                rows.append((tx.shape[1], tx.shape[0], t.filtering, total))
                blocks.append(tx.reshape(-1, 4))
                total += tx.shape[0] * tx.shape[1]
            index[key] = first
            return first

        samp = []
        for m in self.materials:
            row = []
            for key in ("diffuse", "specular", "emissive"):
                sm = m.sampler(key)
                tex = add(sm.textures) if sm.kind in (SAMPLER_TEXTURE, SAMPLER_ERP, SAMPLER_CUBEMAP) else -1
                row.append((sm.kind, tex, tuple(sm.a), tuple(sm.b)))
            samp.append(row)
        env_tex = add(self.env_textures) if self.env_type in (ENV_ERP, ENV_CUBEMAP) else -1
        textures = np.array(rows, np.int64).reshape(-1, 4)
        texels = np.concatenate(blocks).astype(np.float32) if blocks else np.zeros((0, 4), np.float32)
        return textures, texels, samp, env_tex

    @property
    def has_textures(self) -> bool:
        return self.env_type in (ENV_ERP, ENV_CUBEMAP) or any(
            m.samplers and any(v.kind != SAMPLER_COLOR for v in m.samplers.values()) for m in self.materials)

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])

    @property
    def n_prims(self) -> int:
        return int(self.tris.shape[0] + self.spheres.shape[0] + self.planes.shape[0])

    # ------------------------------------------------------------------
    def write_scn(self, directory: str) -> str:
        """Writes ``<name>.scn`` (+ one OBJ per mesh) in the reference's NCF
        format (src/xtcore/proto.h, parseutil.cc:697-822).  Returns the path."""
        os.makedirs(directory, exist_ok=True)
        f = lambda v: repr(float(v))
        v3 = lambda v: "vec3(%s,%s,%s)" % (f(v[0]), f(v[1]), f(v[2]))
        c3 = lambda v: "col3(%s,%s,%s)" % (f(v[0]), f(v[1]), f(v[2]))
        out = ["title = %s" % self.name, "version = 1.0", ""]
        pngs = {}

        def png(t):
            if id(t) not in pngs:
                pngs[id(t)] = "%s_t%02d.png" % (self.name, len(pngs))
                write_png(os.path.join(directory, pngs[id(t)]), t.pixels)
            return pngs[id(t)]

        def sampler_lines(sm, ind):
            if sm.kind == SAMPLER_COLOR:
                return [ind + "type = color", ind + "value = %s" % c3(sm.a)]
            if sm.kind == SAMPLER_GRADIENT:
                return [ind + "type = gradient", ind + "a = %s" % c3(sm.a), ind + "b = %s" % c3(sm.b)]
            if sm.kind == SAMPLER_TEXTURE:
                t = sm.textures[0]
                return [ind + "type = texture", ind + "source = %s" % png(t),
                        ind + "filtering = %s" % ("bilinear" if t.filtering == FILTER_BILINEAR else "nearest"),
                        ind + "flip_x = %s" % ("true" if t.flip_x else "false"),
                        ind + "flip_y = %s" % ("true" if t.flip_y else "false")]
            # the ERP and cubemap textures load with nearest filtering, unflipped
            assert all(t.filtering == FILTER_NEAREST and not t.flip_x and not t.flip_y for t in sm.textures)
            if sm.kind == SAMPLER_ERP:
                return [ind + "type = erp", ind + "source = %s" % png(sm.textures[0])]
            return [ind + "type = cubemap"] + [ind + "%s = %s" % (k, png(t))
                                               for k, t in zip(CUBE_FACE_KEYS, sm.textures)]

        if self.env_type == ENV_ERP:
            out += ["environment = {", "  type = erp", "  config = {",
                    "    source = %s" % png(self.env_textures[0]), "  }", "}"]
        elif self.env_type == ENV_CUBEMAP:
            out += ["environment = {", "  type = cubemap", "  config = {"]
            out += ["    %s = %s" % (k, png(t)) for k, t in zip(CUBE_FACE_KEYS, self.env_textures)]
            out += ["  }", "}"]
        elif self.env_type == ENV_GRADIENT:
            out += ["environment = {", "  type = gradient", "  config = {",
                    "    a = %s" % c3(self.env_a), "    b = %s" % c3(self.env_b), "  }", "}"]
        elif self.env_type == ENV_COLOR:
            out += ["environment = {", "  type = color", "  config = {",
                    "    value = %s" % c3(self.env_a), "  }", "}"]
        out.append("camera = {")
        for cname, cam in [("default", self.camera)] + sorted((self.extra_cameras or {}).items()):
            out += ["  %s = {" % cname, "    type = %s" % CAMERA_NAMES[cam.type],
                    "    position = %s" % v3(cam.position)]
            if cam.type == CAM_PERSPECTIVE:
                out += ["    target = %s" % v3(cam.target), "    up = %s" % v3(cam.up), "    fov = %s" % f(cam.fov)]
                if cam.flength > 0:
                    out += ["    flength = %s" % f(cam.flength), "    aperture = %s" % f(cam.aperture)]
            elif cam.type in (CAM_ERP, CAM_ODS):
                out += ["    orientation = %s" % v3(cam.orientation)]
                if cam.type == CAM_ODS:
                    out += ["    ipd = %s" % f(cam.ipd)]
            out.append("  }")
        out.append("}")
        out.append("geometry = {")
        mesh_i = 0
        mtl_objs = [oi for oi in range(len(self.obj_kind)) if self.mtl_meshes and self.obj_kind[oi] == MESH]
        for oi in range(len(self.obj_kind)):
            if oi in mtl_objs:
                continue
            k, first = int(self.obj_kind[oi]), int(self.obj_first[oi])
            gname = "g%05d" % oi
            uvs = []
            if self.obj_uv_scale is not None and np.any(self.obj_uv_scale[oi] != 0):
                uvs = ["    u_scale = %s" % f(self.obj_uv_scale[oi][0]), "    v_scale = %s" % f(self.obj_uv_scale[oi][1])]
            if k == SPHERE:
                s = self.spheres[first]
                out += ["  %s = {" % gname, "    type = sphere", "    position = %s" % v3(s[:3]),
                        "    radius = %s" % f(s[3])] + uvs + ["  }"]
            elif k == PLANE:
                p = self.planes[first]
                out += ["  %s = {" % gname, "    type = plane", "    normal = %s" % v3(p[:3]),
                        "    distance = %s" % f(p[3])] + uvs + ["  }"]
            else:
                objname = "%s_m%02d.obj" % (self.name, mesh_i)
                self._write_obj(os.path.join(directory, objname), mesh_i, first, int(self.obj_count[oi]))
                mesh_i += 1
                out += ["  %s = {" % gname, "    type = mesh", "    source = %s" % objname] + uvs + ["  }"]
        out.append("}")
        mtl_mats = sorted({int(self.obj_material[oi]) for oi in mtl_objs})
        out.append("material = {")
        for mi, m in enumerate(self.materials):
            if mi in mtl_mats and not any(int(self.obj_material[o]) == mi for o in range(len(self.obj_kind))
                                          if o not in mtl_objs):
                continue
            out += ["  m%05d = {" % mi, "    type = %s" % MATERIAL_NAMES[m.type], "    properties = {",
                    "      samplers = {"]
            for key in ("diffuse", "specular", "emissive"):
                out += ["        %s = {" % key] + sampler_lines(m.sampler(key), "          ") + ["        }"]
            out += ["      }", "      scalars = {", "        reflectance = %s" % f(m.reflectance),
                    "        exponent = %s" % f(m.exponent), "        ior = %s" % f(m.ior),
                    "      }", "    }", "  }"]
        out.append("}")
        out.append("object = {")
        for oi in range(len(self.obj_kind)):
            if oi in mtl_objs:
                continue
            out += ["  o%05d = {" % oi, "    geometry = g%05d" % oi,
                    "    material = m%05d" % int(self.obj_material[oi]), "  }"]
        if mtl_objs:
            # processed after every other object, so its shapes come last in
            # the scene's object map (string-pool ids follow insertion order)
            assert mtl_objs == list(range(len(self.obj_kind) - len(mtl_objs), len(self.obj_kind)))
            objname = self._write_obj_mtl(directory, mtl_objs, png)
            out += ["  o%05d = {" % len(self.obj_kind), "    source = %s" % objname, "    prefix = x", "  }"]
        out.append("}")
        path = os.path.join(directory, self.name + ".scn")
        with open(path, "w") as fh:
            fh.write("\n".join(out) + "\n")
        return path

    def _write_obj_mtl(self, directory: str, objs, png) -> str:
        """One OBJ (a shape per mesh object, each with its usemtl) and its MTL
        library.  A material becomes Emissive when it has an emissive colour or
        texture, else BlinnPhong with Kd / Ks (or map_Kd / map_Ks), Ns and Ni
        (parseutil.cc:604-648); textures load unfiltered and flipped
        horizontally (create_sampler, parseutil.cc:567-585)."""
        f = lambda v: repr(float(v))
        objname, mtlname = self.name + "_ext.obj", self.name + "_ext.mtl"
        mats = sorted({int(self.obj_material[oi]) for oi in objs})
        lines = []
        for mi in mats:
            m = self.materials[mi]
            lines.append("newmtl mat%03d" % mi)
            for key, tag in (("diffuse", "Kd"), ("specular", "Ks"), ("emissive", "Ke")):
                sm = m.sampler(key)
                if sm.kind == SAMPLER_TEXTURE:
                    t = sm.textures[0]
                    assert t.flip_x and not t.flip_y and t.filtering == FILTER_NEAREST
                    lines.append("map_%s %s" % (tag, png(t)))
                else:
                    assert sm.kind == SAMPLER_COLOR
                    lines.append("%s %s %s %s" % ((tag,) + tuple(f(c) for c in sm.a)))
            lines += ["Ns %s" % f(m.exponent), "Ni %s" % f(m.ior), ""]
            emissive = m.sampler("emissive").kind != SAMPLER_COLOR or any(c > 0 for c in m.emissive)
            if emissive:
                assert m.type == EMISSIVE
            else:
                assert m.type == BLINNPHONG and m.reflectance == 0.0
        with open(os.path.join(directory, mtlname), "w") as fh:
            fh.write("\n".join(lines) + "\n")
        out = ["mtllib %s" % mtlname]
        base_v = base_t = 0
        for oi in objs:
            first, count = int(self.obj_first[oi]), int(self.obj_count[oi])
            verts = self.tris[first:first + count].reshape(-1, 3)
            out.append("o shape%05d" % oi)
            out += ["v %r %r %r" % (float(a), float(b), float(c)) for a, b, c in verts.tolist()]
            if self.tri_uvs is not None:
                out += ["vt %r %r" % (float(u), float(v)) for u, v in self.tri_uvs[first:first + count].reshape(-1, 2).tolist()]
            out.append("usemtl mat%03d" % int(self.obj_material[oi]))
            for i in range(count):
                a, b, c = base_v + 3 * i + 1, base_v + 3 * i + 2, base_v + 3 * i + 3
                if self.tri_uvs is not None:
                    t = base_t + 3 * i
                    out.append("f %d/%d %d/%d %d/%d" % (a, t + 1, b, t + 2, c, t + 3))
                else:
                    out.append("f %d %d %d" % (a, b, c))
            base_v += 3 * count
            base_t += 3 * count if self.tri_uvs is not None else 0
        with open(os.path.join(directory, objname), "w") as fh:
            fh.write("\n".join(out) + "\n")
        return objname

    def mesh_obj_path(self, directory: str, mesh_index: int = 0) -> str:
        return os.path.join(directory, "%s_m%02d.obj" % (self.name, mesh_index))

    def _write_obj(self, path: str, mesh_i: int, first: int, count: int) -> None:
        if self.mesh_obj is not None and mesh_i < len(self.mesh_obj) and self.mesh_obj[mesh_i] is not None:
            verts, faces = self.mesh_obj[mesh_i]
        else:
            verts = self.tris[first:first + count].reshape(-1, 3)
            faces = np.arange(count * 3, dtype=np.int64).reshape(-1, 3)
        with open(path, "w") as fh:
            fh.write("".join("v %r %r %r\n" % (float(a), float(b), float(c)) for a, b, c in verts.tolist()))
            if self.tri_uvs is None:
                fh.write("".join("f %d %d %d\n" % (a + 1, b + 1, c + 1) for a, b, c in faces.tolist()))
            else:
                # one texcoord per triangle corner, in face order
                uv = self.tri_uvs[first:first + count].reshape(-1, 2)
                fh.write("".join("vt %r %r\n" % (float(u), float(v)) for u, v in uv.tolist()))
                fh.write("".join("f %d/%d %d/%d %d/%d\n" % (a + 1, 3 * i + 1, b + 1, 3 * i + 2, c + 1, 3 * i + 3)
                                 for i, (a, b, c) in enumerate(faces.tolist())))


# ----------------------------------------------------------------------
def _q(x, step_log2: int) -> np.ndarray:
    """Round to a dyadic grid so the value is an exact float32."""
    s = float(2.0 ** step_log2)
    return (np.round(np.asarray(x, dtype=np.float64) * s) / s).astype(np.float32)


def _qs(x, step_log2: int = 16) -> float:
    return float(_q(np.array([x]), step_log2)[0])


def _objects(kinds, firsts, counts, mats):
    return (np.asarray(kinds, np.int32), np.asarray(firsts, np.int32),
            np.asarray(counts, np.int32), np.asarray(mats, np.int32))


def spheres_scene(n_spheres: int = 64, seed: int = 1, extent: float = 5.0, name: str = None,
                  with_light: bool = True, camera: Camera = None) -> SceneSpec:
    """Ground plane y=0 plus `n_spheres` Lambert spheres: centres uniform in
    [-e,e]x[0.5,4]x[-e,e], radii uniform in [0.2,0.8], albedo uniform in
    [0.1,0.9]^3; a point light at (0,10,0) of intensity 100 (loaded by the
    reference as a radius-0 sphere, parseutil.cc:379-383) and a gradient sky."""
    rng = np.random.default_rng(seed)
    c = np.stack([rng.uniform(-extent, extent, n_spheres), rng.uniform(0.5, 4.0, n_spheres),
                  rng.uniform(-extent, extent, n_spheres)], axis=1)
    r = rng.uniform(0.2, 0.8, n_spheres)
    alb = rng.uniform(0.1, 0.9, (n_spheres, 3))
    sph = np.concatenate([_q(c, 16), _q(r[:, None], 16)], axis=1).astype(np.float32)
    mats = [Material(LAMBERT, diffuse=(0.5, 0.5, 0.5))]
    for i in range(n_spheres):
        a = _q(alb[i], 16)
        mats.append(Material(LAMBERT, diffuse=(float(a[0]), float(a[1]), float(a[2]))))
    kinds, firsts, counts, omat = [PLANE], [0], [1], [0]
    for i in range(n_spheres):
        kinds.append(SPHERE); firsts.append(i); counts.append(1); omat.append(i + 1)
    if with_light:
        sph = np.concatenate([sph, np.array([[0.0, 10.0, 0.0, 0.0]], np.float32)], axis=0)
        mats.append(Material(EMISSIVE, emissive=(100.0, 100.0, 100.0)))
        kinds.append(SPHERE); firsts.append(n_spheres); counts.append(1); omat.append(len(mats) - 1)
    planes = np.array([[0.0, 1.0, 0.0, 0.0]], np.float32)
    k, f, cnt, om = _objects(kinds, firsts, counts, omat)
    cam = camera or Camera((0.0, 6.0, -14.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 60.0)
    if camera is None and extent > 5.0:
        cam = Camera((0.0, 2.5 * extent, -3.0 * extent), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 60.0)
    return SceneSpec(name or ("spheres%d" % n_spheres), sph, planes, np.zeros((0, 3, 3), np.float32),
                     k, f, cnt, om, mats, cam, ENV_GRADIENT, (1.0, 1.0, 1.0), (0.5, 0.7, 1.0))


def phong_scene(seed: int = 51, name: str = "phongscene") -> SceneSpec:
    """Spheres and a plane with Phong and Blinn-Phong materials (phong.cc,
    blinnphong.cc), for the specular lobe (sample.inl:61-90):

    * 16 spheres cycling over {Phong, Blinn-Phong} x reflectance {0.5, 1.0} x
      exponent {8, 256}, colours uniform in [0.1, 0.9]^3;
    * a Blinn-Phong ground plane (reflectance 0.5, exponent 8) and a small
      emissive sphere, under a gradient sky;
    * a Phong sphere (reflectance 1, exponent 256) centred on the camera axis.
      With an odd frame width and height the centre pixel's ray meets it
      head-on, so d.n = 1 and the lobe takes the identity frame; its lobe
      vectors then mostly have vdotr <= 0 or pow(vdotr, 256) below FP64's
      range, and the next ray has no direction."""
    rng = np.random.default_rng(seed)
    mats = [Material(BLINNPHONG, diffuse=(0.5, 0.5, 0.5), specular=(0.8, 0.8, 0.8), reflectance=0.5,
                     exponent=8.0)]
    kinds, firsts, counts, omat = [PLANE], [0], [1], [0]
    sph = []
    for i in range(16):
        gx, gz = i % 4, i // 4
        c = (gx * 2.5 - 3.75 + rng.uniform(-0.3, 0.3), rng.uniform(0.6, 1.2), gz * 2.5 - 1.0 + rng.uniform(-0.3, 0.3))
        r = rng.uniform(0.5, 0.9)
        mtype = PHONG if i % 2 == 0 else BLINNPHONG
        refl = 0.5 if (i // 2) % 2 == 0 else 1.0
        ex = 8.0 if (i // 4) % 2 == 0 else 256.0
        dif, spe = _q(rng.uniform(0.1, 0.9, 3), 16), _q(rng.uniform(0.1, 0.9, 3), 16)
        mats.append(Material(mtype, diffuse=tuple(float(x) for x in dif), specular=tuple(float(x) for x in spe),
                             reflectance=refl, exponent=ex))
        sph.append(list(_q(np.array(c), 16)) + [_qs(r, 16)])
        kinds.append(SPHERE); firsts.append(i); counts.append(1); omat.append(len(mats) - 1)
    # on the camera axis: camera (0, 4, -12) looking at (0, 1, 0)
    mats.append(Material(PHONG, diffuse=(0.5, 0.5, 0.5), specular=(0.9, 0.8, 0.7), reflectance=1.0, exponent=256.0))
    sph.append([0.0, 2.5, -6.0, 0.75])
    kinds.append(SPHERE); firsts.append(16); counts.append(1); omat.append(len(mats) - 1)
    mats.append(Material(EMISSIVE, emissive=(6.0, 5.5, 5.0)))
    sph.append([2.0, 4.5, 3.0, 0.5])
    kinds.append(SPHERE); firsts.append(17); counts.append(1); omat.append(len(mats) - 1)
    planes = np.array([[0.0, 1.0, 0.0, 0.0]], np.float32)
    k, f, cnt, om = _objects(kinds, firsts, counts, omat)
    cam = Camera((0.0, 4.0, -12.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 60.0)
    return SceneSpec(name, np.array(sph, np.float32), planes, np.zeros((0, 3, 3), np.float32), k, f, cnt, om,
                     mats, cam, ENV_GRADIENT, (1.0, 1.0, 1.0), (0.5, 0.7, 1.0))


def _value_noise(x: np.ndarray, z: np.ndarray, lattice: np.ndarray) -> np.ndarray:
    """Value noise with smoothstep interpolation on a periodic random lattice."""
    L = lattice.shape[0]
    xi = np.floor(x); zi = np.floor(z)
    fx = x - xi; fz = z - zi
    sx = fx * fx * (3 - 2 * fx); sz = fz * fz * (3 - 2 * fz)
    i0 = xi.astype(np.int64) % L; j0 = zi.astype(np.int64) % L
    i1 = (i0 + 1) % L; j1 = (j0 + 1) % L
    a = lattice[i0, j0]; b = lattice[i1, j0]; c = lattice[i0, j1]; d = lattice[i1, j1]
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def terrain_mesh(grid: int = 708, seed: int = 2, half: float = 50.0, amplitude: float = 8.0,
                 octaves: int = 6, base_freq: float = 1.0 / 16.0, offset=(0.0, 0.0)):
    """Height field over [-half,half]^2 on a grid x grid vertex lattice:
    height = sum_{o<octaves} amplitude * 2^-o * valuenoise(2^o * base_freq * (x,z)).
    Returns (verts (V,3) float32, faces (F,3) int64) with 2 triangles per quad in
    row-major order."""
    rng = np.random.default_rng(seed)
    lattices = [rng.uniform(-1.0, 1.0, (64, 64)) for _ in range(octaves)]
    lin = np.linspace(-half, half, grid)
    X, Z = np.meshgrid(lin + offset[0], lin + offset[1], indexing="xy")
    H = np.zeros_like(X)
    for o in range(octaves):
        fq = (2.0 ** o) * base_freq
        H += amplitude * (2.0 ** -o) * _value_noise(X * fq, Z * fq, lattices[o])
    verts = np.stack([_q(X, 16), _q(H, 16), _q(Z, 16)], axis=-1).reshape(-1, 3).astype(np.float32)
    idx = np.arange(grid * grid, dtype=np.int64).reshape(grid, grid)
    a = idx[:-1, :-1].ravel(); b = idx[:-1, 1:].ravel(); c = idx[1:, :-1].ravel(); d = idx[1:, 1:].ravel()
    faces = np.empty((a.size * 2, 3), np.int64)
    # counter-clockwise seen from above: face normals point up (+y)
    faces[0::2] = np.stack([a, c, b], axis=1)
    faces[1::2] = np.stack([b, c, d], axis=1)
    return verts, faces


def uv_scene(seed: int = 6, name: str = "uvscene") -> SceneSpec:
    """Texture-coordinate paths of every primitive kind: 24 spheres (half with
    u/v scales), a ground plane with u/v scales, and a terrain patch whose
    triangles carry OBJ texcoords; some materials emissive.  For the normal, uv
    and emission integrators."""
    rng = np.random.default_rng(seed)
    base = spheres_scene(24, seed=seed, extent=5.0, name=name, with_light=False)
    verts, faces = terrain_mesh(12, seed + 1, half=3.0, amplitude=0.5, octaves=2, offset=(0.0, 2.0))
    verts = verts + np.array([0.0, 0.25, 2.0], np.float32)
    tris = verts[faces].astype(np.float32)
    uv = np.stack([(verts[:, 0] + 3.0) / 6.0, (verts[:, 2] - 2.0 + 3.0) / 6.0], axis=1)
    tri_uvs = _q(uv[faces], 12).astype(np.float32)
    n_obj = len(base.obj_kind)
    scale = np.zeros((n_obj + 1, 2), np.float32)
    scale[0] = (0.25, 0.5)                                # the plane
    for oi in range(1, n_obj, 2):                         # every other sphere
        scale[oi] = _q(rng.uniform(0.5, 2.0, 2), 8)
    scale[n_obj] = (0.0, 0.0)                             # the mesh (triangles use tc only)
    mats = list(base.materials)
    for i in range(1, len(mats), 3):                      # every third sphere glows
        e = _q(rng.uniform(0.2, 3.0, 3), 8)
        mats[i] = Material(EMISSIVE, emissive=(float(e[0]), float(e[1]), float(e[2])))
    mats.append(Material(LAMBERT, diffuse=(0.3, 0.6, 0.3), emissive=(0.5, 0.25, 0.125)))
    kinds = np.concatenate([base.obj_kind, [MESH]]).astype(np.int32)
    firsts = np.concatenate([base.obj_first, [0]]).astype(np.int32)
    counts = np.concatenate([base.obj_count, [tris.shape[0]]]).astype(np.int32)
    omat = np.concatenate([base.obj_material, [len(mats) - 1]]).astype(np.int32)
    return SceneSpec(name, base.spheres, base.planes, tris, kinds, firsts, counts, omat, mats, base.camera,
                     ENV_GRADIENT, base.env_a, base.env_b, mesh_obj=[(verts, faces)], obj_uv_scale=scale,
                     tri_uvs=tri_uvs)


def textured_scene(env: str = "erp", seed: int = 9, name: str = None) -> SceneSpec:
    """Every sampler kind on every primitive kind: the uv scene's spheres,
    ground plane and texcoord-carrying terrain patch with 2D textures (nearest
    and bilinear, flipped and not, RGB and RGBA, odd sizes), ERP, cubemap and
    gradient material samplers on diffuse, specular and emissive, and an ERP
    or cubemap environment."""
    rng = np.random.default_rng(seed)
    base = uv_scene(seed=6, name=name or ("tex_" + env))
    img = lambda h, w, c=3: rng.integers(0, 256, (h, w, c), dtype=np.uint8)
    t_near = Texture(img(5, 7), FILTER_NEAREST)
    t_bil = Texture(img(6, 9, 4), FILTER_BILINEAR, flip_x=True)
    t_flip = Texture(img(8, 8), FILTER_BILINEAR, flip_y=True)
    t_wide = Texture(img(4, 16), FILTER_NEAREST, flip_x=True, flip_y=True)
    m_erp = Texture(img(9, 17))
    m_cube = tuple(Texture(img(4 + i % 3, 5)) for i in range(6))
    samplers = [
        {"diffuse": Sampler(SAMPLER_TEXTURE, textures=(t_near,))},
        {"emissive": Sampler(SAMPLER_TEXTURE, textures=(t_bil,))},
        {"diffuse": Sampler(SAMPLER_ERP, textures=(m_erp,)), "emissive": Sampler(SAMPLER_ERP, textures=(m_erp,))},
        {"emissive": Sampler(SAMPLER_CUBEMAP, textures=m_cube)},
        {"diffuse": Sampler(SAMPLER_GRADIENT, (0.25, 0.5, 1.0), (1.0, 0.5, 0.125)),
         "specular": Sampler(SAMPLER_TEXTURE, textures=(t_wide,)),
         "emissive": Sampler(SAMPLER_GRADIENT, (0.5, 0.25, 0.0), (0.0, 0.75, 1.0))},
        {"emissive": Sampler(SAMPLER_TEXTURE, textures=(t_flip,))},
    ]
    mats = []
    for i, m in enumerate(base.materials):
        mats.append(dataclasses.replace(m, samplers=samplers[i % len(samplers)]))
    # u/v scales of at least 1 keep every sphere texcoord finite (a scale below
    # 1 drives asin out of its domain: NaN texcoords, covered by the uv scenes)
    uvs = base.obj_uv_scale.copy()
    small = (uvs > 0) & (uvs < 1)
    uvs[small] = _q(1.0 / uvs[small], 8)
    spec = dataclasses.replace(base, materials=mats, obj_uv_scale=uvs)
    if env == "erp":
        spec.env_type, spec.env_textures = ENV_ERP, (Texture(img(16, 32)),)
    else:
        spec.env_type, spec.env_textures = ENV_CUBEMAP, tuple(Texture(img(6 + i, 6 + i)) for i in range(6))
    return spec


def mtl_scene(seed: int = 12, name: str = "mtlscene") -> SceneSpec:
    """Meshes from one OBJ with an MTL library behind the loader's external
    object path: BlinnPhong shapes with Kd / Ks colours or map_Kd / map_Ks
    textures and Emissive shapes with Ke or map_Ke, with OBJ texcoords; spheres
    and a ground plane from the .scn before them; gradient sky."""
    rng = np.random.default_rng(seed)
    base = spheres_scene(12, seed=seed, extent=5.0, name=name, with_light=False)
    img = lambda h, w: rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    tex = [Texture(img(6, 5), FILTER_NEAREST, flip_x=True), Texture(img(4, 9), FILTER_NEAREST, flip_x=True),
           Texture(img(8, 8), FILTER_NEAREST, flip_x=True)]
    tris, uvs, kinds, firsts, counts, omat = [], [], [], [], [], []
    mats = list(base.materials)
    col = lambda: tuple(float(v) for v in _q(rng.uniform(0.1, 0.9, 3), 8))
    specs = [Material(BLINNPHONG, diffuse=col(), specular=col(), exponent=16.0, ior=1.5),
             Material(BLINNPHONG, diffuse=col(), specular=col(), exponent=64.0, ior=1.25,
                      samplers={"diffuse": Sampler(SAMPLER_TEXTURE, textures=(tex[0],))}),
             Material(BLINNPHONG, diffuse=col(), exponent=8.0, ior=1.0,
                      samplers={"specular": Sampler(SAMPLER_TEXTURE, textures=(tex[1],))}),
             # Emissive materials from MTL get no scalars (ior and exponent read 0)
             Material(EMISSIVE, emissive=(2.0, 1.5, 0.5), ior=0.0),
             Material(EMISSIVE, samplers={"emissive": Sampler(SAMPLER_TEXTURE, textures=(tex[2],))}, ior=0.0)]
    n = 0
    for k, m in enumerate(specs):
        verts, faces = terrain_mesh(6, seed + k, half=1.0, amplitude=0.25, octaves=2, offset=(0.0, 0.0))
        verts = verts + np.array([-4.0 + 2.0 * k, 1.5, 2.0 + (k % 2)], np.float32)
        t = verts[faces].astype(np.float32)
        uv = np.stack([(verts[:, 0] - verts[:, 0].min()) / 2.0, (verts[:, 2] - verts[:, 2].min()) / 2.0], axis=1)
        tris.append(t)
        uvs.append(_q(uv[faces], 12).astype(np.float32))
        mats.append(m)
        kinds.append(MESH); firsts.append(n); counts.append(t.shape[0]); omat.append(len(mats) - 1)
        n += t.shape[0]
    n_base = len(base.obj_kind)
    scale = np.zeros((n_base + len(specs), 2), np.float32)
    scale[n_base:] = 1.0            # ISurface's default (surface.cc:8): the OBJ meshes keep it
    return SceneSpec(name, base.spheres, base.planes, np.concatenate(tris), np.concatenate([base.obj_kind, kinds]),
                     np.concatenate([base.obj_first, firsts]).astype(np.int32),
                     np.concatenate([base.obj_count, counts]).astype(np.int32),
                     np.concatenate([base.obj_material, omat]).astype(np.int32), mats, base.camera,
                     ENV_GRADIENT, base.env_a, base.env_b, obj_uv_scale=scale, tri_uvs=np.concatenate(uvs),
                     mtl_meshes=True)


def grid_for_tris(n_tris: int) -> int:
    return 1 + int(round(math.sqrt(n_tris / 2.0)))


def terrain_scene(n_tris: int = 999_698, seed: int = 2, name: str = None) -> SceneSpec:
    """Config-2 terrain: ~n_tris triangles (708^2 grid gives 999,698) of 6-octave
    value noise, amplitude 8, over [-50,50]^2, one Lambert mesh, gradient sky."""
    grid = grid_for_tris(n_tris)
    verts, faces = terrain_mesh(grid, seed)
    tris = verts[faces]
    k, f, cnt, om = _objects([MESH], [0], [tris.shape[0]], [0])
    cam = Camera((0.0, 30.0, -75.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0)
    return SceneSpec(name or ("terrain%d" % tris.shape[0]), np.zeros((0, 4), np.float32),
                     np.zeros((0, 4), np.float32), tris.astype(np.float32), k, f, cnt, om,
                     [Material(LAMBERT, diffuse=(0.6, 0.5, 0.4))], cam, ENV_GRADIENT,
                     (1.0, 1.0, 1.0), (0.5, 0.7, 1.0), mesh_obj=[(verts, faces)])


def hairball_tris(n_tris: int = 2_000_000, seed: int = 3, edge: float = 0.01, radius: float = 1.0,
                  center=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Equilateral triangles of the given edge, centroids uniform in a ball,
    orientations from uniform random quaternions (Shoemake 1992)."""
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(n_tris, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    rad = radius * rng.uniform(0.0, 1.0, n_tris) ** (1.0 / 3.0)
    cen = u * rad[:, None] + np.asarray(center)[None, :]
    r1, r2, r3 = rng.uniform(0, 1, (3, n_tris))
    q = np.stack([np.sqrt(1 - r1) * np.sin(2 * np.pi * r2), np.sqrt(1 - r1) * np.cos(2 * np.pi * r2),
                  np.sqrt(r1) * np.sin(2 * np.pi * r3), np.sqrt(r1) * np.cos(2 * np.pi * r3)], axis=1)
    x, y, z, w = q.T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                  np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                  np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], axis=1)
    cr = edge / math.sqrt(3.0)
    ang = np.array([0.0, 2 * np.pi / 3, 4 * np.pi / 3])
    local = np.stack([cr * np.cos(ang), cr * np.sin(ang), np.zeros(3)], axis=1)   # (3,3)
    v = cen[:, None, :] + np.einsum("nij,kj->nki", R, local)
    scale_log2 = 22 if (radius + abs(max(center, key=abs)) + edge) < 2.0 else 16
    return _q(v, scale_log2).astype(np.float32)


def hairball_scene(n_tris: int = 2_000_000, seed: int = 3, name: str = None) -> SceneSpec:
    """Config-3 hairball: n_tris equilateral triangles (edge 0.01) with centroids
    uniform in the unit ball, one Lambert mesh, gradient sky."""
    tris = hairball_tris(n_tris, seed)
    k, f, cnt, om = _objects([MESH], [0], [tris.shape[0]], [0])
    cam = Camera((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0)
    return SceneSpec(name or ("hairball%d" % n_tris), np.zeros((0, 4), np.float32),
                     np.zeros((0, 4), np.float32), tris, k, f, cnt, om,
                     [Material(LAMBERT, diffuse=(0.8, 0.8, 0.8))], cam, ENV_GRADIENT,
                     (1.0, 1.0, 1.0), (0.5, 0.7, 1.0))


def precision_scene(scale: float = 1.0, seed: int = 5) -> SceneSpec:
    """Config-5 scene: 8 displaced terrain tiles + 4 hairballs (8M triangles at
    scale 1), Phong / Blinn-Phong materials with exponent uniform in [8,256] and
    reflectance 0.5, one emissive sphere and one 200-triangle emissive mesh."""
    rng = np.random.default_rng(seed)
    tile_tris = max(2, int(500_000 * scale))
    hb_tris = max(1, int(1_000_000 * scale))
    chunks, kinds, firsts, counts, omat, mats = [], [], [], [], [], []
    first = 0
    for t in range(8):
        ox, oz = (t % 4) * 100.0 - 150.0, (t // 4) * 100.0 - 50.0
        verts, faces = terrain_mesh(grid_for_tris(tile_tris), seed * 100 + t, offset=(ox, oz))
        tri = verts[faces]
        chunks.append(tri); kinds.append(MESH); firsts.append(first); counts.append(tri.shape[0])
        mats.append(Material(PHONG if t % 2 == 0 else BLINNPHONG, diffuse=(0.6, 0.55, 0.5),
                             specular=(0.9, 0.9, 0.9), reflectance=0.5,
                             exponent=_qs(rng.uniform(8, 256), 8)))
        omat.append(len(mats) - 1); first += tri.shape[0]
    for h in range(4):
        c = ((h % 2) * 100.0 - 50.0, 12.0, (h // 2) * 60.0 - 30.0)
        tri = hairball_tris(hb_tris, seed * 1000 + h, edge=0.1, radius=8.0, center=c)
        chunks.append(tri); kinds.append(MESH); firsts.append(first); counts.append(tri.shape[0])
        mats.append(Material(BLINNPHONG if h % 2 == 0 else PHONG, diffuse=(0.7, 0.7, 0.7),
                             specular=(1.0, 1.0, 1.0), reflectance=0.5,
                             exponent=_qs(rng.uniform(8, 256), 8)))
        omat.append(len(mats) - 1); first += tri.shape[0]
    # 200-triangle emissive mesh: a 10x10 quad grid above the scene
    g = np.linspace(-20.0, 20.0, 11)
    X, Z = np.meshgrid(g, g, indexing="xy")
    lv = np.stack([X, np.full_like(X, 60.0), Z], -1).reshape(-1, 3)
    idx = np.arange(121).reshape(11, 11)
    a = idx[:-1, :-1].ravel(); b = idx[:-1, 1:].ravel(); cc = idx[1:, :-1].ravel(); d = idx[1:, 1:].ravel()
    lf = np.empty((200, 3), np.int64); lf[0::2] = np.stack([a, cc, b], 1); lf[1::2] = np.stack([b, cc, d], 1)
    ltri = _q(lv, 16)[lf]
    chunks.append(ltri); kinds.append(MESH); firsts.append(first); counts.append(200)
    mats.append(Material(EMISSIVE, emissive=(20.0, 20.0, 20.0))); omat.append(len(mats) - 1)
    first += 200
    sph = np.array([[30.0, 40.0, 0.0, 6.0]], np.float32)
    kinds.append(SPHERE); firsts.append(0); counts.append(1)
    mats.append(Material(EMISSIVE, emissive=(40.0, 38.0, 30.0))); omat.append(len(mats) - 1)
    tris = np.concatenate(chunks, axis=0).astype(np.float32)
    k, f, cnt, om = _objects(kinds, firsts, counts, omat)
    cam = Camera((0.0, 60.0, -160.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0)
    return SceneSpec("precision8m" if scale == 1.0 else "precision_s%g" % scale, sph,
                     np.zeros((0, 4), np.float32), tris, k, f, cnt, om, mats, cam, ENV_NONE)


# ----------------------------------------------------------------------
JOBSTREAM_SCENES = [("terrain10k", 10_000), ("terrain50k", 50_000), ("terrain200k", 200_000),
                    ("terrain500k", 500_000), ("terrain1m", 1_000_000), ("hairball2m", 2_000_000),
                    ("spheres64", 64), ("spheres4096", 4096)]


def jobstream_scene(name: str, scale: float = 1.0) -> SceneSpec:
    """The 8 resident scenes of the served job stream (terrain and hairball
    generators at 10k..2M triangles, plus 64- and 4096-sphere scenes)."""
    n = dict(JOBSTREAM_SCENES)[name]
    if name.startswith("terrain"):
        return terrain_scene(max(8, int(n * scale)), seed=40 + int(math.log2(n)), name=name)
    if name.startswith("hairball"):
        return hairball_scene(max(8, int(n * scale)), seed=43, name=name)
    if n == 64:
        return spheres_scene(64, seed=44, name=name)
    return spheres_scene(n, seed=45, extent=40.0, name=name)


@dataclasses.dataclass
class Job:
    job_id: int
    scene: int          # index into the resident scene list
    width: int
    height: int
    spp: int
    depth: int
    arrival_s: float
    seed: int


def job_stream(n_jobs: int = 512, seed: int = 4, rate_hz: float = 50.0, n_scenes: int = 8,
               resolutions=(128, 256, 512, 1024), spps=(1, 4, 16, 64), depth: int = 4) -> List[Job]:
    """Poisson arrivals at `rate_hz`; resolution and spp uniform over the given
    sets, scene uniform over the resident scenes, pathtracer depth 4."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, n_jobs)
    t = np.cumsum(gaps) - gaps[0]
    jobs = []
    for i in range(n_jobs):
        r = int(rng.choice(resolutions)); s = int(rng.choice(spps)); sc = int(rng.integers(0, n_scenes))
        jobs.append(Job(i, sc, r, r, s, depth, float(t[i]), int(rng.integers(1, 2 ** 62))))
    return jobs
