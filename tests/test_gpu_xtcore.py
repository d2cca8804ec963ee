"""The GPU integrator inside XTracer's own host: xtgpu-xtcore loads a .scn with
io::scn::load, runs IIntegrator::render() (OpenMP tile loop, produce/pop
contract) with xtcore::integrator::gpu::Integrator and assembles the tiles.

* The frame equals, bit for bit, the C ABI's render of the generator's scene
  (same seed): flattening and the tile plumbing lose nothing.
* Depth and stencil agree with the reference's CPU integrators run by the same
  binary on the same loaded Scene (primitive ties and grazing hits aside)."""
import numpy as np
import pytest

from xtracer_b200 import scenes, xtgpu
from tests import xtcore_host as xh

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not xh.available(), reason="xtgpu-xtcore not built (needs the XTracer sources)")]

NAMES = {xtgpu.STENCIL: "stencil", xtgpu.DEPTH: "depth", xtgpu.AO: "ao", xtgpu.PATHTRACER: "pathtracer",
         xtgpu.NORMAL: "normal", xtgpu.UV: "uv", xtgpu.EMISSION: "emission", xtgpu.WIREFRAME: "wireframe"}


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


@pytest.fixture(scope="module")
def written(tmp_path_factory):
    d = tmp_path_factory.mktemp("scn")
    specs = [scenes.spheres_scene(64, seed=1, name="s64"), scenes.terrain_scene(5_000, seed=2, name="t5k"),
             scenes.hairball_scene(3_000, seed=3, name="h3k"), scenes.uv_scene(6)]
    return [(s, s.write_scn(str(d))) for s in specs], d


def render_host(scn, kind, w, h, spp, rdepth, out, *extra):
    r = xh.run("render", scn, NAMES[kind], w, h, spp, rdepth, out, *extra)
    assert r.returncode == 0, r.stdout + r.stderr
    return xh.read_frame(out)


@pytest.mark.parametrize("kind, spp, rdepth, extra", [
    (xtgpu.STENCIL, 2, 1, ()), (xtgpu.DEPTH, 1, 1, ()), (xtgpu.AO, 4, 1, ()),
    (xtgpu.AO, 4, 1, ("--ao-distance", "0.25")), (xtgpu.PATHTRACER, 4, 4, ()),
    (xtgpu.PATHTRACER, 3, 4, ("--q8", "--seed", "7", "--tile", "16")),
    (xtgpu.PATHTRACER, 2, 4, ("--w8",)),
    (xtgpu.NORMAL, 3, 1, ()), (xtgpu.UV, 3, 1, ()), (xtgpu.EMISSION, 3, 1, ()), (xtgpu.WIREFRAME, 2, 1, ())])
def test_integrator_in_host_equals_c_abi(written, kind, spp, rdepth, extra):
    specs, d = written
    fmt = xtgpu.NODES_Q8 if "--q8" in extra else (xtgpu.NODES_W8 if "--w8" in extra else xtgpu.NODES_FP32)
    seed = int(extra[extra.index("--seed") + 1]) if "--seed" in extra else 1
    aod = float(extra[extra.index("--ao-distance") + 1]) if "--ao-distance" in extra else 100.0
    for spec, scn in specs:
        got = render_host(scn, kind, 80, 56, spp, rdepth, d / ("%s.bin" % spec.name), *extra)
        sc = xtgpu.Scene(spec, node_formats=(fmt,))
        ref, _ = sc.render(kind, 80, 56, spp=spp, rdepth=rdepth, ao_max_distance=aod, seed=seed, node_format=fmt)
        sc.close()
        assert np.array_equal(got, ref, equal_nan=True), "%s %s differs through the xtcore host" % (spec.name,
                                                                                                    NAMES[kind])


@pytest.mark.parametrize("kind", [xtgpu.STENCIL, xtgpu.DEPTH])
def test_integrator_in_host_matches_reference_cpu_integrator(written, kind):
    specs, d = written
    for spec, scn in specs[:2]:
        gpu = render_host(scn, kind, 64, 48, 1, 1, d / "g.bin")
        cpu = render_host(scn, kind, 64, 48, 1, 1, d / "c.bin", "--cpu", "--threads", "4")
        if kind == xtgpu.STENCIL:
            bad = np.any(gpu != cpu, axis=2)
        else:
            bad = np.abs(gpu[..., 0] - cpu[..., 0]) > 1e-5 * np.maximum(np.abs(cpu[..., 0]), 1e-30)
            bad |= gpu[..., 3] != cpu[..., 3]
        # a mismatch is a hit/miss or primitive disagreement on a grazing ray
        assert bad.sum() <= 2, "%s %s: %d pixels differ" % (spec.name, NAMES[kind], bad.sum())


@pytest.mark.parametrize("kind, spp, rdepth, scene", [(xtgpu.PATHTRACER, 4, 4, 0), (xtgpu.UV, 3, 1, 3),
                                                       (xtgpu.DEPTH, 1, 1, 1), (xtgpu.STENCIL, 3, 1, 2)])
def test_png_exr_output_match_reference_writers(written, kind, spp, rdepth, scene):
    """The frame written through the GPU quantiser and this library's PNG and
    EXR writers decodes to exactly what XTracer's own writers (nimg::io::save,
    lib/nimg/img.cc:72-179) produce from the same assembled frame: PNG pixels
    bit for bit (values above 1 clamped, NaN channels 0), EXR floats bit for bit."""
    from PIL import Image
    specs, d = written
    spec, scn = specs[scene]
    p = {k: str(d / ("%s_%d.%s" % (k.split(".")[0], kind, k.split(".")[1])))
         for k in ("own.png", "ref.png", "own.exr", "ref.exr")}
    r = xh.run("render", scn, NAMES[kind], 72, 40, spp, rdepth, d / "o.bin", "--png", p["own.png"],
               "--ref-png", p["ref.png"], "--exr", p["own.exr"], "--ref-exr", p["ref.exr"])
    assert r.returncode == 0, r.stdout + r.stderr
    a = np.asarray(Image.open(p["own.png"]).convert("RGBA"))
    b = np.asarray(Image.open(p["ref.png"]).convert("RGBA"))
    assert a.shape == b.shape == (40, 72, 4)
    assert np.array_equal(a, b)
    ea, eb = xh.read_exr(p["own.exr"]), xh.read_exr(p["ref.exr"])
    assert sorted(ea) == sorted(eb) == ["B", "G", "R"]
    for c in "BGR":
        assert np.array_equal(ea[c], eb[c], equal_nan=True)
    frame = xh.read_frame(d / "o.bin")
    assert np.array_equal(ea["R"], frame[..., 0], equal_nan=True)


@pytest.mark.parametrize("cam, w, h", [
    (scenes.Camera((0.0, 3.0, -12.0), (0.0, 1.5, 0.0), (0.0, 1.0, 0.0), 50.0, flength=11.0, aperture=0.75), 48, 40),
    (scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_ERP, orientation=(0.25, -0.5, 0.125)), 96, 48),
    (scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_ODS, orientation=(0.0, 0.75, 0.0), ipd=0.125), 64, 64),
    (scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_CUBEMAP), 24, 144)], ids=["dof", "erp", "ods", "cubemap"])
def test_cameras_and_aa_in_host_equal_c_abi(tmp_path, cam, w, h):
    """Every camera type of a .scn and the context's aa level (grid
    distribution) reach the GPU through the xtcore host unchanged."""
    spec = scenes.spheres_scene(64, seed=1, name="hostcam", camera=cam)
    scn = spec.write_scn(str(tmp_path))
    for kind, spp, aa in ((xtgpu.DEPTH, 2, 2), (xtgpu.AO, 2, 3)):
        got = render_host(scn, kind, w, h, spp, 1, tmp_path / "f.bin", "--aa", str(aa), "--ao-distance", "0.5")
        sc = xtgpu.Scene(spec)
        ref, _ = sc.render(kind, w, h, spp=spp, rdepth=1, ao_max_distance=0.5, seed=1, aa=aa)
        sc.close()
        assert np.array_equal(got, ref, equal_nan=True), NAMES[kind]


def test_random_distribution_in_host_equals_c_abi(tmp_path):
    """params_t::sample_distribution = RANDOM reaches the GPU: aa jittered
    positions per pixel, the frame equal to the C ABI's with the same seed;
    aa = 0 with it writes no pixel, as the CPU integrators do."""
    spec = scenes.spheres_scene(64, seed=1, name="hostrnd")
    scn = spec.write_scn(str(tmp_path))
    sc = xtgpu.Scene(spec)
    for kind, spp, aa in ((xtgpu.DEPTH, 2, 3), (xtgpu.AO, 2, 5), (xtgpu.STENCIL, 1, 1)):
        got = render_host(scn, kind, 48, 40, spp, 1, tmp_path / "f.bin", "--aa", str(aa), "--random",
                          "--ao-distance", "0.5", "--seed", "9")
        ref, _ = sc.render(kind, 48, 40, spp=spp, rdepth=1, ao_max_distance=0.5, seed=9, aa=aa,
                           distribution=xtgpu.SAMPLES_RANDOM)
        assert np.array_equal(got, ref, equal_nan=True), NAMES[kind]
    sc.close()
    gpu = render_host(scn, xtgpu.STENCIL, 32, 24, 1, 1, tmp_path / "g0.bin", "--aa", "0", "--random")
    cpu = render_host(scn, xtgpu.STENCIL, 32, 24, 1, 1, tmp_path / "c0.bin", "--aa", "0", "--random", "--cpu")
    assert np.array_equal(gpu, cpu)


def test_aa_zero_writes_no_pixel(written):
    """aa = 0: antialiasing::produce gives the tiles no samples (aa.cc:9), so
    the frame keeps what tile->init wrote, as with the CPU integrators."""
    specs, d = written
    spec, scn = specs[0]
    gpu = render_host(scn, xtgpu.STENCIL, 32, 24, 1, 1, d / "g0.bin", "--aa", "0")
    cpu = render_host(scn, xtgpu.STENCIL, 32, 24, 1, 1, d / "c0.bin", "--aa", "0", "--cpu")
    assert np.array_equal(gpu, cpu)


@pytest.mark.parametrize("env", ["erp", "cubemap"])
def test_textured_scene_in_host_equals_c_abi(tmp_path, env):
    """PNG textures, filtering and flip keys, ERP / cubemap samplers and
    environments loaded by XTracer's own loader render, through the xtcore
    host, to the C ABI's bits for the generator's scene."""
    spec = scenes.textured_scene(env)
    scn = spec.write_scn(str(tmp_path))
    for kind, spp, rdepth, aa in ((xtgpu.EMISSION, 2, 1, 2), (xtgpu.PATHTRACER, 4, 4, 1)):
        got = render_host(scn, kind, 64, 48, spp, rdepth, tmp_path / "f.bin", "--aa", str(aa))
        sc = xtgpu.Scene(spec)
        ref, _ = sc.render(kind, 64, 48, spp=spp, rdepth=rdepth, seed=1, aa=aa)
        sc.close()
        assert np.array_equal(got, ref), NAMES[kind]


def test_obj_mtl_scene_in_host_equals_c_abi(tmp_path):
    """Meshes, materials and textures from an OBJ + MTL, loaded by XTracer's
    external object path, render through the xtcore host to the C ABI's bits
    for the generator's scene."""
    spec = scenes.mtl_scene()
    scn = spec.write_scn(str(tmp_path))
    for kind, spp, rdepth in ((xtgpu.EMISSION, 2, 1), (xtgpu.PATHTRACER, 4, 4)):
        got = render_host(scn, kind, 64, 48, spp, rdepth, tmp_path / "f.bin")
        sc = xtgpu.Scene(spec)
        ref, _ = sc.render(kind, 64, 48, spp=spp, rdepth=rdepth, seed=1)
        sc.close()
        assert np.array_equal(got, ref), NAMES[kind]


def test_camera_switch_in_host(tmp_path):
    """The context renders through another camera of the same scene: the GPU
    integrator follows it (camera re-upload, geometry kept), matching the C
    ABI's render through that camera and the CPU integrator."""
    import dataclasses
    spec = scenes.spheres_scene(64, seed=1, name="twocams")
    alt = scenes.Camera((0.5, 2.0, 0.25), type=scenes.CAM_ERP, orientation=(0.0, 0.5, 0.0))
    spec = dataclasses.replace(spec, extra_cameras={"alt": alt})
    scn = spec.write_scn(str(tmp_path))
    got = render_host(scn, xtgpu.DEPTH, 64, 32, 2, 1, tmp_path / "g.bin", "--then-camera", "alt")
    cpu = render_host(scn, xtgpu.DEPTH, 64, 32, 2, 1, tmp_path / "c.bin", "--then-camera", "alt", "--cpu",
                      "--threads", "2")
    sc = xtgpu.Scene(dataclasses.replace(spec, camera=alt))
    ref, _ = sc.render(xtgpu.DEPTH, 64, 32, spp=2)
    sc.close()
    assert np.array_equal(got, ref)
    D = np.abs(cpu[..., 0].astype(np.float64))
    assert np.mean(np.abs(got[..., 0] - cpu[..., 0]) <= 1e-5 * D * np.maximum(1.0, D) + 1e-7) >= 0.99
