"""Fixed-batch measurement of the extend kernel (closest-hit traversal).

One scene of the served job stream; primary rays of its camera, then a batch of
first-bounce rays, cosine-distributed around the face normal at each primary
hit (primary rays that missed stay in the batch).  Times xtgpu_trace on the
bounce batch with CUDA events and reports Mrays/s, nodes and primitives per ray,
algorithmic bytes per ray and achieved GB/s; the extend kernel's ncu captures
run this script.

    python -m xtracer_b200.profile_extend --scene hairball2m --rays 1048576 --fmt q8 --iters 5
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math

import numpy as np


def camera_rays(spec, w, h):
    """Pixel-centre pinhole rays (Perspective::get_primary_ray, aa = 1), FP64."""
    cam = spec.camera
    pos = np.array(cam.position, np.float64)
    rz = np.array(cam.target, np.float64) - pos
    rz /= np.linalg.norm(rz)
    rx = np.cross(np.array(cam.up, np.float64), rz)
    rx /= np.linalg.norm(rx)
    ry = np.cross(rx, rz)
    ry /= np.linalg.norm(ry)
    ys, xs = np.mgrid[0:h, 0:w]
    dx = 2.0 * (xs.ravel() + 0.5) / w - 1.0
    dy = (2.0 * (ys.ravel() + 0.5) / h - 1.0) / (w / h)
    dz = 1.0 / math.tan(cam.fov * 0.017453292519943 / 2.0)
    d = rx[None] * dx[:, None] + ry[None] * dy[:, None] + rz[None] * dz
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.broadcast_to(pos, d.shape).copy(), d


def normals_at(spec, prim, p):
    nt, ns = spec.n_tris, spec.spheres.shape[0]
    n = np.zeros_like(p)
    t = prim < nt
    if t.any():
        v = spec.tris[prim[t]].astype(np.float64)
        n[t] = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    s = (prim >= nt) & (prim < nt + ns)
    if s.any():
        sp = spec.spheres[prim[s] - nt].astype(np.float64)
        n[s] = p[s] - sp[:, :3]
    pl = prim >= nt + ns
    if pl.any():
        n[pl] = spec.planes[prim[pl] - nt - ns, :3]
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)


def cosine_dirs(n, rng):
    u, v = rng.random(n.shape[0]), rng.random(n.shape[0])
    r, phi = np.sqrt(u), 2 * np.pi * v
    local = np.stack([r * np.cos(phi), np.sqrt(1 - u), r * np.sin(phi)], 1)
    a = np.where(np.abs(n[:, :1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    x = np.cross(a, n)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    z = np.cross(x, n)
    return x * local[:, :1] + n * local[:, 1:2] + z * local[:, 2:3]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="hairball2m")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--rays", type=int, default=1 << 20)
    ap.add_argument("--fmt", default="q8", choices=["fp32", "q8", "w8"])
    ap.add_argument("--iters", type=int, default=5)
    args = ap.parse_args()
    import torch
    from . import scenes, xtgpu
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    fmt = {"fp32": xtgpu.NODES_FP32, "q8": xtgpu.NODES_Q8, "w8": xtgpu.NODES_W8}[args.fmt]
    spec = scenes.jobstream_scene(args.scene, args.scale)
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8), leaf_size=1)
    side = int(math.ceil(math.sqrt(args.rays)))
    o, d = camera_rays(spec, side, side)
    o, d = o[:args.rays], d[:args.rays]
    n = o.shape[0]
    hits = sc.intersection(o.astype(np.float32), d.astype(np.float32), node_format=fmt)
    hit = hits["prim"] != 0xffffffff
    p = o + d * np.where(hit, hits["t"], 0.0)[:, None]
    nrm = normals_at(spec, hits["prim"][hit].astype(np.int64), p[hit])
    nrm *= -np.sign(np.sum(nrm * d[hit], axis=1, keepdims=True))   # face the incoming ray
    rng = np.random.default_rng(1)
    o2, d2 = o.copy(), d.copy()
    o2[hit] = p[hit] + nrm * 1e-4 * (1.0 + np.abs(p[hit]).max(axis=1, keepdims=True))
    d2[hit] = cosine_dirs(nrm, rng)
    org = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    dr = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    org[:, :3] = torch.from_numpy(o2.astype(np.float32)).cuda()
    dr[:, :3] = torch.from_numpy(d2.astype(np.float32)).cuda()
    dr[:, 3] = float("inf")
    hits_d = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    L = xtgpu.lib()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    sh = xtgpu.stream_handle(stream)
    counts = (C.c_uint64 * 2)()
    xtgpu.check(L.xtgpu_trace_counts(sc.handle, n, ptr(org), ptr(dr), ptr(hits_d), fmt, counts, sh))
    vn, vp = counts[0] / n, counts[1] / n
    node_bytes = xtgpu.NODE_BYTES[fmt]
    bpr = 32 + 16 + vn * node_bytes + vp * 48
    times = []
    for _ in range(args.iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        xtgpu.check(L.xtgpu_trace(sc.handle, n, ptr(org), ptr(dr), ptr(hits_d), fmt, sh))
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    print(json.dumps({"scene": args.scene, "fmt": args.fmt, "rays": n, "bounce_fraction": float(hit.mean()),
                      "ms": ms, "mrays": n / ms / 1e3, "nodes_per_ray": vn, "prims_per_ray": vp,
                      "bytes_per_ray": bpr, "achieved_gbs": n * bpr / ms / 1e6,
                      "tuning": {k: getattr(xtgpu.get_tuning(), k) for k, _ in xtgpu.Tuning._fields_}}))


if __name__ == "__main__":
    main()
