"""The xtcore-side Scene flattener (xtracer_b200/xtcore/gpu_integrator.cc) on
scenes loaded by XTracer's own io::scn::load: the description it hands the C
ABI equals the generator's, object by object, and what the GPU path cannot
render is refused with a reason.  CPU only: flattening makes no CUDA call."""
import os

import numpy as np
import pytest

from xtracer_b200 import scenes
from tests import xtcore_host as xh

pytestmark = pytest.mark.skipif(not xh.available(), reason="xtgpu-xtcore not built (needs the XTracer sources)")


def flatten(spec, tmp_path):
    scn = spec.write_scn(str(tmp_path))
    out = tmp_path / "flat.bin"
    r = xh.run("flatten", scn, out)
    assert r.returncode == 0, r.stderr
    return xh.read_flat(out)


@pytest.mark.parametrize("make", [lambda: scenes.spheres_scene(64, seed=1, name="s64"),
                                  lambda: scenes.terrain_scene(5_000, seed=2, name="t5k"),
                                  lambda: scenes.hairball_scene(3_000, seed=3, name="h3k"),
                                  lambda: scenes.precision_scene(scale=0.002, seed=5),
                                  lambda: scenes.uv_scene(6)])
def test_flattened_scene_equals_generator(make, tmp_path):
    spec = make()
    d = flatten(spec, tmp_path)
    for key in ("obj_kind", "obj_first", "obj_count"):
        assert np.array_equal(d[key], getattr(spec, key)), key
    assert np.array_equal(d["spheres"], spec.spheres)
    assert np.array_equal(d["planes"], spec.planes)
    # mesh triangles come out of each Mesh's octree items, in OBJ face order
    assert np.array_equal(d["tris"], spec.tris)
    assert d["tri_normals"] is None
    uvs = spec.obj_uv_scale if spec.obj_uv_scale is not None else np.zeros((len(spec.obj_kind), 2), np.float32)
    assert np.array_equal(d["obj_uv_scale"], uvs)
    if spec.tri_uvs is None:
        assert d["tri_uvs"] is None          # the Triangle constructor's texcoords
    else:
        assert np.array_equal(d["tri_uvs"], spec.tri_uvs)
    assert d["env_type"] == spec.env_type
    assert np.array_equal(d["env_a"], np.float32(spec.env_a))
    if spec.env_type == scenes.ENV_GRADIENT:
        assert np.array_equal(d["env_b"], np.float32(spec.env_b))
    cam = spec.camera
    assert np.array_equal(d["camera"], np.float32(list(cam.position) + list(cam.target) + list(cam.up) + [cam.fov]))
    assert d["camera_type"] == scenes.CAM_PERSPECTIVE and d["camera_flength"] == 0.0
    for oi in range(len(spec.obj_kind)):
        t, row = d["materials"][d["obj_material"][oi]]
        m = spec.materials[spec.obj_material[oi]]
        assert t == m.type, oi
        assert np.array_equal(row, xh.material_row(m)), oi


SCN_HEAD = """title = t
version = 1.0
camera = {
  default = {
    type = thin-lens
    position = vec3(0,1,-5)
    target = vec3(0,0,0)
    up = vec3(0,1,0)
    fov = 60
%s  }
}
geometry = {
  g0 = {
    type = %s
    position = vec3(0,0,0)
    radius = 1
  }
}
material = {
  m0 = {
    type = lambert
    properties = {
      samplers = {
        diffuse = {
%s
        }
      }
    }
  }
}
object = {
  o0 = {
    geometry = g0
    material = m0
  }
}
"""
COLOUR = "          type = color\n          value = col3(0.5,0.5,0.5)"
TEXTURE = "          type = texture\n          source = missing.png"


@pytest.mark.parametrize("extra, geom, sampler, why", [
    ("", "sphere", TEXTURE, "failed to load"),
])
def test_unsupported_features_are_refused(tmp_path, extra, geom, sampler, why):
    scn = tmp_path / "u.scn"
    scn.write_text(SCN_HEAD % (extra, geom, sampler))
    r = xh.run("flatten", scn, tmp_path / "f.bin")
    assert r.returncode == 1
    assert why in r.stderr


def test_point_geometry_is_a_zero_radius_sphere(tmp_path):
    """The loader makes `point` geometry a Sphere of radius 0
    (parseutil.cc:379-383); the flattener passes it on as such."""
    scn = tmp_path / "p.scn"
    scn.write_text((SCN_HEAD % ("", "point", COLOUR)).replace("    radius = 1\n", ""))
    r = xh.run("flatten", scn, tmp_path / "f.bin")
    assert r.returncode == 0, r.stderr
    d = xh.read_flat(tmp_path / "f.bin")
    assert d["obj_kind"].tolist() == [scenes.SPHERE]
    assert d["spheres"].tolist() == [[0.0, 0.0, 0.0, 0.0]]


@pytest.mark.parametrize("cam", [
    scenes.Camera((0.5, 3.0, -12.0), (0.0, 1.5, 0.0), (0.0, 1.0, 0.0), 50.0, flength=11.0, aperture=0.75),
    scenes.Camera((0.25, 1.0, -0.5), type=scenes.CAM_ERP, orientation=(0.1, -0.4, 0.2)),
    scenes.Camera((0.0, 1.0, 0.25), type=scenes.CAM_ODS, orientation=(0.0, 0.3, 0.0), ipd=0.125),
    scenes.Camera((1.0, 0.5, -2.0), type=scenes.CAM_CUBEMAP),
], ids=["thin-lens-dof", "erp", "ods", "cubemap"])
def test_every_camera_type_is_flattened(cam, tmp_path):
    """Thin-lens (with depth of field), ERP, ODS and cubemap cameras of a .scn
    reach the C ABI's camera with the loader's values (parseutil.cc camera
    fields: position, orientation, ipd, flength, aperture)."""
    spec = scenes.spheres_scene(16, seed=4, name="cams")
    spec.camera = cam
    d = flatten(spec, tmp_path)
    assert d["camera_type"] == cam.type
    assert np.array_equal(d["camera"][:3], np.float32(cam.position))
    if cam.type == scenes.CAM_PERSPECTIVE:
        assert np.array_equal(d["camera"][3:], np.float32(list(cam.target) + list(cam.up) + [cam.fov]))
        assert d["camera_flength"] == np.float32(cam.flength)
        assert d["camera_aperture"] == np.float32(cam.aperture)
    if cam.type in (scenes.CAM_ERP, scenes.CAM_ODS):
        assert np.array_equal(d["camera_orientation"], np.float32(cam.orientation))
    if cam.type == scenes.CAM_ODS:
        assert d["camera_ipd"] == np.float32(cam.ipd)


def _texture_of(d, idx):
    w, h, filt, off = d["textures"][idx]
    return d["texels"][off:off + w * h].reshape(h, w, 4), filt


@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_scene_samplers_are_flattened(env, tmp_path):
    """Every material's diffuse, specular and emissive sampler and the
    environment reach the C ABI as the loader built them: kinds, colours,
    and the texels of each texture (PNG loaded by stbi, /255, flips applied)
    with its filtering; a cubemap's six faces in CUBEMAP_FACE order."""
    spec = scenes.textured_scene(env)
    d = flatten(spec, tmp_path)
    assert d["samplers"] is not None
    for oi in range(len(spec.obj_kind)):
        m = spec.materials[spec.obj_material[oi]]
        for ch, key in enumerate(("diffuse", "specular", "emissive")):
            kind, tex, a, b = d["samplers"][3 * d["obj_material"][oi] + ch]
            want = m.sampler(key)
            assert kind == want.kind, (oi, key)
            if kind in (scenes.SAMPLER_COLOR, scenes.SAMPLER_GRADIENT):
                assert np.array_equal(a, np.float32(want.a)), (oi, key)
            if kind == scenes.SAMPLER_GRADIENT:
                assert np.array_equal(b, np.float32(want.b)), (oi, key)
            for k, t in enumerate(want.textures):
                texels, filt = _texture_of(d, tex + k)
                assert np.array_equal(texels, t.texels()), (oi, key, k)
                assert filt == t.filtering
    assert d["env_type"] == (scenes.ENV_ERP if env == "erp" else scenes.ENV_CUBEMAP)
    for k, t in enumerate(spec.env_textures):
        texels, filt = _texture_of(d, d["env_texture"] + k)
        assert np.array_equal(texels, t.texels()), ("env", k)


def test_obj_mtl_scene_is_flattened(tmp_path):
    """Meshes from an OBJ with an MTL library (the loader's external object
    path): the flattened objects, triangles, texcoords, materials and samplers
    equal the generator's; the OBJ's shapes follow the .scn objects."""
    spec = scenes.mtl_scene()
    d = flatten(spec, tmp_path)
    for key in ("obj_kind", "obj_first", "obj_count"):
        assert np.array_equal(d[key], getattr(spec, key)), key
    assert np.array_equal(d["tris"], spec.tris)
    assert np.array_equal(d["tri_uvs"], spec.tri_uvs)
    assert np.array_equal(d["obj_uv_scale"], spec.obj_uv_scale)
    for oi in range(len(spec.obj_kind)):
        m = spec.materials[spec.obj_material[oi]]
        t, row = d["materials"][d["obj_material"][oi]]
        assert t == m.type, oi
        assert row[9] == m.reflectance and row[10] == m.exponent and row[11] == m.ior, oi
        for ch, key in enumerate(("diffuse", "specular", "emissive")):
            kind, tex, a, b = d["samplers"][3 * d["obj_material"][oi] + ch]
            want = m.sampler(key)
            assert kind == want.kind, (oi, key)
            if kind == scenes.SAMPLER_COLOR:
                assert np.array_equal(a, np.float32(want.a)), (oi, key)
            else:
                texels, filt = _texture_of(d, tex)
                assert np.array_equal(texels, want.textures[0].texels()) and filt == scenes.FILTER_NEAREST
