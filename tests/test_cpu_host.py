"""Host-side checks that need no GPU: the C ABI library loads and exports
every entry point include/xtgpu.h declares, argument checks reject bad input
before any device work, the scene generators produce exact float32 inputs, and
the CPU LBVH replica builds a valid Karras hierarchy."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po
from xtracer_b200 import scenes, xtgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "xtgpu.h")).read()
    return sorted(set(re.findall(r"XTGPU_API\s+[\w\s\*]+?\b(xtgpu_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", xtgpu.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (xtgpu_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = xtgpu.lib()
    for n in names:
        assert getattr(L, n) is not None
    assert set(xtgpu.SIGNATURES) | {"xtgpu_last_error", "xtgpu_version"} == set(names)


def test_library_is_sm100a():
    out = subprocess.run(["strings", xtgpu.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out or "compute_100a" in out or xtgpu.lib().xtgpu_version().decode().endswith("(sm_100a)")


def test_invalid_arguments_are_rejected_without_device_work():
    L = xtgpu.lib()
    out = C.c_void_p()
    assert L.xtgpu_scene_create(None, None, C.byref(out)) == 1
    d = xtgpu.SceneDesc()
    d.n_tris = 3            # triangles without an array
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    assert b"NULL arrays" in L.xtgpu_last_error()
    d = xtgpu.SceneDesc()   # a sphere that belongs to no object
    sph = np.zeros(4, np.float32)
    d.n_spheres = 1
    d.spheres = sph.ctypes.data_as(C.c_void_p)
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    assert b"no object" in L.xtgpu_last_error()
    assert L.xtgpu_bvh_build(None, None, None) == 1
    assert L.xtgpu_render(None, None, None, None, None) == 1
    assert L.xtgpu_trace(None, 4, None, None, None, 0, None) == 1
    assert L.xtgpu_service_create(None, None, C.byref(out)) == 1
    o = xtgpu.ServiceOpts(1 << 20, 0, 0, 0, 1, 1, 0, 0, 0, 0)   # max_jobs 0
    assert L.xtgpu_service_create(C.byref(o), None, C.byref(out)) == 1
    for wif in (-1, 5):   # waves in flight outside 0..XTGPU_MAX_WAVES_IN_FLIGHT
        o = xtgpu.ServiceOpts(1 << 20, 8, 0, 0, 1, 1, 0, 0, 0, 0, wif)
        assert L.xtgpu_service_create(C.byref(o), None, C.byref(out)) == 1
    assert L.xtgpu_scene_destroy(None) == 0


def test_generated_scenes_are_exact_float32():
    for spec in (scenes.spheres_scene(64, seed=1), scenes.terrain_scene(5_000, seed=2),
                 scenes.hairball_scene(5_000, seed=3)):
        for a in (spec.spheres, spec.planes, spec.tris):
            a64 = a.astype(np.float64)
            # dyadic grid: every value round-trips through its shortest repr
            for v in a64.ravel()[:2000]:
                assert float(repr(float(v))) == v and np.float32(v) == v
        assert spec.obj_kind.size == spec.obj_first.size == spec.obj_count.size == spec.obj_material.size


def test_terrain_sizes_and_orientation():
    spec = scenes.terrain_scene(999_698, seed=2)
    assert spec.n_tris == 999_698
    t = spec.tris[:1000].astype(np.float64)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    assert np.all(n[:, 1] > 0), "terrain faces wound counter-clockwise seen from above"
    assert spec.tris[:, :, 0].min() == -50.0 and spec.tris[:, :, 0].max() == 50.0


def test_hairball_geometry():
    t = scenes.hairball_tris(20_000, seed=3).astype(np.float64)
    e = np.linalg.norm(t[:, 1] - t[:, 0], axis=1)
    assert np.allclose(e, 0.01, atol=1e-5)
    c = t.mean(axis=1)
    assert np.linalg.norm(c, axis=1).max() <= 1.0 + 1e-5


def test_job_stream_is_seeded():
    a = scenes.job_stream(512, seed=4)
    b = scenes.job_stream(512, seed=4)
    assert [(j.scene, j.width, j.spp, j.arrival_s) for j in a] == [(j.scene, j.width, j.spp, j.arrival_s) for j in b]
    assert {j.width for j in a} == {128, 256, 512, 1024} and {j.spp for j in a} == {1, 4, 16, 64}
    assert all(j.depth == 4 for j in a)
    assert all(x.arrival_s <= y.arrival_s for x, y in zip(a, a[1:]))


@pytest.mark.parametrize("n_sph", [1, 2, 3, 64, 4096])
def test_cpu_lbvh_replica_is_a_valid_karras_tree(n_sph):
    spec = scenes.spheres_scene(n_sph, seed=5, with_light=False)
    L = po.lib()
    L.xo_lbvh_build.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p] + [C.c_void_p] * 4
    n = n_sph
    keys = np.zeros(n, np.uint32); order = np.zeros(n, np.uint32)
    left = np.zeros(max(n - 1, 1), np.int32); right = np.zeros(max(n - 1, 1), np.int32)
    sph = np.ascontiguousarray(spec.spheres.reshape(-1), np.float32)
    L.xo_lbvh_build(0, None, n, sph.ctypes.data_as(C.c_void_p), *[a.ctypes.data_as(C.c_void_p)
                                                                  for a in (keys, order, left, right)])
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(order), np.arange(n))
    if n > 1:
        left, right = left[:n - 1], right[:n - 1]
        inner = np.concatenate([left[left >= 0], right[right >= 0]])
        leaves = np.concatenate([~left[left < 0], ~right[right < 0]])
        assert np.array_equal(np.sort(inner), np.arange(1, n - 1))
        assert np.array_equal(np.sort(leaves), np.arange(n))


def test_bad_textures_and_cameras_are_rejected_without_device_work():
    """Texture tables, sampler texture indices, environment textures and camera
    types are checked on the host before any device allocation."""
    L = xtgpu.lib()
    out = C.c_void_p()

    def desc():
        d = xtgpu.SceneDesc()
        d.env_texture = -1
        return d

    texels = np.zeros((6, 4), np.float32)
    tex = (xtgpu.Texture * 1)()
    tex[0].width, tex[0].height, tex[0].filtering, tex[0].offset = 3, 3, 0, 0   # 9 texels > 6
    d = desc()
    d.n_textures, d.textures, d.n_texels = 1, C.cast(tex, C.c_void_p), 6
    d.texels = texels.ctypes.data_as(C.c_void_p)
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    assert b"texture 0" in L.xtgpu_last_error()
    tex[0].width, tex[0].height, tex[0].filtering = 2, 3, 7                      # bad filtering
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    tex[0].filtering = 1
    d.env_type, d.env_texture = 4, 0                                               # cubemap needs 6
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    assert b"environment texture" in L.xtgpu_last_error()
    d.env_type = 3
    mats = (xtgpu.Material * 1)()
    sam = (xtgpu.SamplerDesc * 3)()
    sam[0].kind, sam[0].texture = 2, 1                                             # texture 1 of 1
    d.n_materials, d.materials, d.mat_samplers = 1, C.cast(mats, C.c_void_p), C.cast(sam, C.c_void_p)
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    assert b"material sampler 0" in L.xtgpu_last_error()
    d = desc()
    d.camera.type = 9
    assert L.xtgpu_scene_create(C.byref(d), None, C.byref(out)) == 1
    assert b"camera" in L.xtgpu_last_error()


def test_scene_update_arguments_are_checked_without_device_work():
    L = xtgpu.lib()
    d = xtgpu.SceneDesc()
    assert L.xtgpu_scene_update(None, C.byref(d), 1, None) == 1
    assert L.xtgpu_service_update_scene(None, 0) == 1


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every structure of include/xtgpu.h that the Python binding mirrors has
    the header's size and field offsets (compiled with gcc here)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    from xtracer_b200 import xtgpu
    pairs = {"xtgpu_material": xtgpu.Material, "xtgpu_camera": xtgpu.CameraDesc, "xtgpu_texture": xtgpu.Texture,
             "xtgpu_sampler": xtgpu.SamplerDesc, "xtgpu_scene_desc": xtgpu.SceneDesc,
             "xtgpu_bvh_opts": xtgpu.BvhOpts, "xtgpu_bvh_info": xtgpu.BvhInfo, "xtgpu_hit": xtgpu.Hit,
             "xtgpu_render_params": xtgpu.RenderParams, "xtgpu_service_opts": xtgpu.ServiceOpts,
             "xtgpu_service_stats": xtgpu.ServiceStats, "xtgpu_tuning": xtgpu.Tuning,
             "xtgpu_job_desc": xtgpu.JobDesc, "xtgpu_job_status": xtgpu.JobStatus}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "xtgpu.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in py._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", inc, str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                 text=True).stdout.splitlines())
    for cname, py in pairs.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for f in py._fields_:
            assert int(out["%s.%s" % (cname, f[0])]) == getattr(py, f[0]).offset, (cname, f[0])
