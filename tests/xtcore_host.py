"""Helpers for the tests of the xtcore-side GPU integrator: the xtgpu-xtcore
front end (XTracer's host code + the GPU integrator, built by
xtracer_b200/xtcore/xtcore.mk) and readers for its output files."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "xtracer_b200", "_build", "xtgpu-xtcore")


def available() -> bool:
    return os.access(BINARY, os.X_OK)


def run(*args, timeout=600):
    return subprocess.run([BINARY] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)


def read_flat(path):
    """The flattened scene description written by `xtgpu-xtcore flatten`."""
    b = open(path, "rb").read()
    off = 0

    def take(dt, n):
        nonlocal off
        a = np.frombuffer(b, dt, n, off)
        off += a.nbytes
        return a

    no, ns, npl, nt, nm, hn, env, hu = (int(v) for v in take(np.int32, 8))
    d = {"env_type": env}
    for key in ("obj_kind", "obj_first", "obj_count", "obj_material"):
        d[key] = take(np.int32, no)
    d["spheres"] = take(np.float32, 4 * ns).reshape(-1, 4)
    d["planes"] = take(np.float32, 4 * npl).reshape(-1, 4)
    d["tris"] = take(np.float32, 9 * nt).reshape(-1, 3, 3)
    d["tri_normals"] = take(np.float32, 9 * nt).reshape(-1, 3, 3) if hn else None
    d["obj_uv_scale"] = take(np.float32, 2 * no).reshape(-1, 2)
    d["tri_uvs"] = take(np.float32, 6 * nt).reshape(-1, 3, 2) if hu else None
    d["materials"] = []
    for _ in range(nm):
        t = int(take(np.int32, 1)[0])
        d["materials"].append((t, take(np.float32, 12)))
    d["env_a"], d["env_b"] = take(np.float32, 3), take(np.float32, 3)
    d["camera"] = take(np.float32, 10)
    d["camera_type"] = int(take(np.int32, 1)[0])
    d["camera_orientation"] = take(np.float32, 3)
    d["camera_ipd"], d["camera_flength"], d["camera_aperture"] = (float(v) for v in take(np.float32, 3))
    n_tex, has_samp, d["env_texture"] = (int(v) for v in take(np.int32, 3))
    d["textures"] = []
    for _ in range(n_tex):
        w, h, filt = (int(v) for v in take(np.int32, 3))
        d["textures"].append((w, h, filt, int(take(np.int64, 1)[0])))
    n_texels = int(take(np.int64, 1)[0])
    d["texels"] = take(np.float32, 4 * n_texels).reshape(-1, 4)
    d["samplers"] = None
    if has_samp:
        d["samplers"] = []
        for _ in range(3 * len(d["materials"])):
            kind, tex = (int(v) for v in take(np.int32, 2))
            d["samplers"].append((kind, tex, take(np.float32, 3), take(np.float32, 3)))
    assert off == len(b), "trailing bytes in the flattened scene"
    return d


def read_frame(path):
    """The frame written by `xtgpu-xtcore render`: (H, W, 4) float32."""
    b = open(path, "rb").read()
    w, h = (int(v) for v in np.frombuffer(b, np.int32, 2))
    return np.frombuffer(b, np.float32, 4 * w * h, 8).reshape(h, w, 4)


def material_row(m):
    return np.array(list(m.diffuse) + list(m.specular) + list(m.emissive) + [m.reflectance, m.exponent, m.ior],
                    np.float32)


def read_exr(path):
    """Channels of an uncompressed scanline OpenEXR file: {name: (H, W) float32}."""
    b = open(path, "rb").read()
    assert b[:4] == bytes([0x76, 0x2f, 0x31, 0x01])
    off = 8
    attrs = {}
    while b[off] != 0:
        e = b.index(b"\0", off); name = b[off:e].decode(); off = e + 1
        e = b.index(b"\0", off); typ = b[off:e].decode(); off = e + 1
        size = int(np.frombuffer(b, np.int32, 1, off)[0]); off += 4
        attrs[name] = (typ, b[off:off + size]); off += size
    off += 1
    assert attrs["compression"][1][0] == 0, "compressed EXR"
    x0, y0, x1, y1 = (int(v) for v in np.frombuffer(attrs["dataWindow"][1], np.int32))
    w, h = x1 - x0 + 1, y1 - y0 + 1
    chl, names, p = attrs["channels"][1], [], 0
    while chl[p] != 0:
        e = chl.index(b"\0", p); names.append(chl[p:e].decode()); p = e + 1 + 16
    offsets = np.frombuffer(b, np.uint64, h, off)
    out = {n: np.zeros((h, w), np.float32) for n in names}
    for o in offsets:
        o = int(o)
        y = int(np.frombuffer(b, np.int32, 1, o)[0]) - y0
        data = np.frombuffer(b, np.float32, w * len(names), o + 8)
        for k, n in enumerate(names):
            out[n][y] = data[k * w:(k + 1) * w]
    return out
