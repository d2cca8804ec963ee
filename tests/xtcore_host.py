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
