"""The depth integrator's raygraph on the GPU (depth/integrator.cc:43-51,
util/raygraph.cc:8-75): per sample the ray origin, the hit point and the
pixel's colour after the sample, exported as the GUI exports it.

* Against the reference's own PLY (tests/golden/raygraph.npz): the same
  header and edges; vertices equal up to the FP32 trace (origins exact; hit
  points and colours within 1e-5 relative, the colour being the depth fold
  1/log(t), whose relative error grows with |depth|).
* The frame rendered with the raygraph is the plain depth frame.
* Through the xtcore host (tiles' bundles, the reference's own writer): the
  same file as the C ABI's records through xtgpu_write_raygraph_ply."""
import importlib.util
import os

import numpy as np
import pytest

from xtracer_b200 import scenes, xtgpu
from tests import xtcore_host as xh

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


def _case():
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    return mg.raygraph_case()


def parse_ply(text):
    lines = text.splitlines()
    end = lines.index("end_header")
    head = lines[:end + 1]
    nv = int([l for l in head if l.startswith("element vertex")][0].split()[-1])
    verts = np.array([[float(v) for v in l.split()] for l in lines[end + 1:end + 1 + nv]]).reshape(-1, 6)
    edges = lines[end + 1 + nv:]
    return head, verts, edges


def close(a, b, rel):
    return np.abs(a - b) <= rel * np.maximum(1.0, np.abs(b)) * np.maximum(1.0, np.abs(b)) + 1e-5 * np.abs(b) + 2e-6


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_W8])
def test_raygraph_vs_reference_golden(tmp_path, fmt):
    spec, w, h, spp, aa = _case()
    g = np.load(os.path.join(GOLD, "raygraph.npz"))
    sc = xtgpu.Scene(spec, node_formats=(fmt,), leaf_size=1)
    img, rec = sc.render_raygraph(w, h, spp=spp, aa=aa, node_format=fmt)
    plain, _ = sc.render(xtgpu.DEPTH, w, h, spp=spp, aa=aa, node_format=fmt)
    sc.close()
    assert np.array_equal(img, plain)
    path = str(tmp_path / "rg.ply")
    xtgpu.save_raygraph_ply(path, rec)
    gh, gv, ge = parse_ply(open(path).read())
    rh, rv, re_ = parse_ply(g["ply"].tobytes().decode())
    assert gh == rh and ge == re_
    origin, hit = gv[0::2], gv[1::2]
    r_origin, r_hit = rv[0::2], rv[1::2]
    assert np.array_equal(origin, r_origin)
    ok = close(hit[:, :3], r_hit[:, :3], 0.0).all(axis=1) & close(hit[:, 3:], r_hit[:, 3:], 1e-5).all(axis=1)
    assert ok.mean() >= 0.998, (ok.mean(), np.argwhere(~ok)[:5].ravel())


@pytest.mark.skipif(not xh.available(), reason="xtgpu-xtcore not built (needs the XTracer sources)")
def test_raygraph_through_xtcore_host(tmp_path):
    """GPU integrator inside XTracer's tile loop: the tiles' bundles, exported
    by XTracer's own writer, equal the C ABI's records written by
    xtgpu_write_raygraph_ply, and agree with the CPU depth integrator's."""
    spec, w, h, spp, aa = _case()
    scn = spec.write_scn(str(tmp_path))
    r = xh.run("render", scn, "depth", w, h, spp, 1, tmp_path / "g.bin", "--aa", aa, "--raygraph", tmp_path / "g.ply")
    assert r.returncode == 0, r.stdout + r.stderr
    r = xh.run("render", scn, "depth", w, h, spp, 1, tmp_path / "c.bin", "--aa", aa, "--raygraph",
               tmp_path / "c.ply", "--cpu", "--threads", "2")
    assert r.returncode == 0, r.stdout + r.stderr
    sc = xtgpu.Scene(spec)
    _, rec = sc.render_raygraph(w, h, spp=spp, aa=aa)
    sc.close()
    xtgpu.save_raygraph_ply(str(tmp_path / "abi.ply"), rec)
    host = open(tmp_path / "g.ply").read()
    assert host == open(tmp_path / "abi.ply").read()
    gh, gv, ge = parse_ply(host)
    ch, cv, ce = parse_ply(open(tmp_path / "c.ply").read())
    assert gh == ch and ge == ce
    ok = close(gv[1::2, :3], cv[1::2, :3], 0.0).all(axis=1) & close(gv[1::2, 3:], cv[1::2, 3:], 1e-5).all(axis=1)
    assert ok.mean() >= 0.998
