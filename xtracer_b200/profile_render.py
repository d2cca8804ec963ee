"""One frame of one served-stream scene through xtgpu_render, for kernel
captures of the whole wavefront (camera, extend, shade, accumulate) on full
waves.  Renders the job `--iters` times after one warm-up render and reports
the device time per frame and Mrays/s; the shade kernel's ncu captures run
this script.

    python -m xtracer_b200.profile_render --scene terrain200k --size 1024 --spp 4
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="terrain200k")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--spp", type=int, default=4)
    ap.add_argument("--depth", type=int, default=4)
    ap.add_argument("--fmt", default="w8", choices=["fp32", "q8", "w8"])
    ap.add_argument("--iters", type=int, default=3)
    args = ap.parse_args()
    import torch
    from . import scenes, xtgpu
    torch.cuda.set_device(0)
    fmt = {"fp32": xtgpu.NODES_FP32, "q8": xtgpu.NODES_Q8, "w8": xtgpu.NODES_W8}[args.fmt]
    spec = scenes.jobstream_scene(args.scene, args.scale)
    sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, fmt), leaf_size=1)
    w = h = args.size
    frame = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    p = xtgpu.RenderParams(xtgpu.PATHTRACER, w, h, args.spp, args.depth, 100.0, 7, fmt, 0, 0, 0, 0, 1)
    import ctypes as C
    rays = C.c_uint64()
    L = xtgpu.lib()
    stream = torch.cuda.current_stream()

    def render():
        xtgpu.check(L.xtgpu_render(sc.handle, C.byref(p), C.c_void_p(frame.data_ptr()), C.byref(rays),
                                   C.c_void_p(stream.cuda_stream)))

    render()
    times = []
    for _ in range(args.iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        render()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = min(times)
    print(json.dumps({"scene": args.scene, "size": w, "spp": args.spp, "fmt": args.fmt, "ms": ms,
                      "rays": int(rays.value), "mrays": rays.value / ms / 1e3}))
    sc.close()


if __name__ == "__main__":
    main()
