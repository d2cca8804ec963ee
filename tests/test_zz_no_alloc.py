"""xtgpu_render_tile_noalloc, the rendering entry point that allocates nothing
(for callers that cannot allocate device memory at render time, such as a
render_tile on XTracer's OpenMP tile threads where a cudaMalloc would stall the
device), against xtgpu_render on the same rectangle.  Two calls in a row share
the static scratch array, so the second must not see the first's leftovers.
Collected last on purpose: it must also pass alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from xtracer_b200 import scenes, xtgpu

pytestmark = pytest.mark.gpu


def _noalloc(sc, integ, w, h, spp, rect, out, rdepth=4, md=2.0, seed=5):
    x0, y0, x1, y1 = rect
    p = xtgpu.RenderParams(integ, w, h, spp, rdepth, md, seed, xtgpu.NODES_FP32, x0, y0, x1, y1)
    rays = C.c_uint64()
    st = xtgpu.lib().xtgpu_render_tile_noalloc(sc.handle, C.byref(p), C.c_void_p(out.data_ptr()), C.byref(rays),
                                               None)
    return st, int(rays.value)


def test_noalloc_tile_equals_render_on_two_calls():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    spec = scenes.spheres_scene(64, seed=1, name="noalloc")
    sc = xtgpu.Scene(spec)
    w, h = 64, 48
    rect = (16, 8, 48, 40)   # a 32x32 tile
    for integ, spp in ((xtgpu.PATHTRACER, 16), (xtgpu.AO, 64), (xtgpu.DEPTH, 2), (xtgpu.STENCIL, 1)):
        ref, ref_rays = sc.render(integ, w, h, spp=spp, rdepth=4, ao_max_distance=2.0, seed=5, rect=rect)
        out = torch.empty((32, 32, 4), dtype=torch.float32, device="cuda")
        for call in range(2):
            out.fill_(-7.0)
            st, rays = _noalloc(sc, integ, w, h, spp, rect, out)
            assert st == 0, xtgpu.lib().xtgpu_last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            # same kernels, same random stream: the tolerance of the other
            # determinism tests, bit-identical
            assert np.array_equal(got, ref), "call %d, integrator %d" % (call, integ)
            assert rays == ref_rays
    sc.close()


def test_noalloc_rejects_requests_beyond_its_array():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    sc = xtgpu.Scene(scenes.spheres_scene(8, seed=2, name="noalloc_big"))
    out = torch.empty((64, 64, 4), dtype=torch.float32, device="cuda")
    st, _ = _noalloc(sc, xtgpu.PATHTRACER, 64, 64, 17, (0, 0, 64, 64), out)   # 69632 paths > 65536
    assert st == 4
    assert b"65536" in xtgpu.lib().xtgpu_last_error()
    st, _ = _noalloc(sc, xtgpu.PATHTRACER, 64, 64, 16, (0, 0, 64, 64), out)   # exactly 65536 paths
    assert st == 0
    sc.close()


def test_noalloc_concurrent_host_threads():
    """Tiles rendered at once from several host threads (XTracer's OpenMP tile
    loop), each on its own stream, equal the same tiles rendered one by one:
    the calls take turns on the shared scratch array."""
    import threading

    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    sc = xtgpu.Scene(scenes.terrain_scene(20_000, seed=2, name="noalloc_mt"))
    w, h = 128, 64
    rects = [(x, y, x + 32, y + 32) for y in (0, 32) for x in (0, 32, 64, 96)]
    refs = [sc.render(xtgpu.PATHTRACER, w, h, spp=8, rdepth=4, seed=5, rect=r)[0] for r in rects]
    outs = [torch.empty((32, 32, 4), dtype=torch.float32, device="cuda") for _ in rects]
    streams = [torch.cuda.Stream() for _ in rects]
    status = [None] * len(rects)

    def work(k):
        torch.cuda.set_device(0)
        x0, y0, x1, y1 = rects[k]
        p = xtgpu.RenderParams(xtgpu.PATHTRACER, w, h, 8, 4, 2.0, 5, xtgpu.NODES_FP32, x0, y0, x1, y1)
        rays = C.c_uint64()
        status[k] = xtgpu.lib().xtgpu_render_tile_noalloc(sc.handle, C.byref(p), C.c_void_p(outs[k].data_ptr()),
                                                          C.byref(rays), C.c_void_p(streams[k].cuda_stream))

    for rep in range(3):
        for o in outs:
            o.fill_(-7.0)
        torch.cuda.synchronize()
        threads = [threading.Thread(target=work, args=(k,)) for k in range(len(rects))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize()
        assert status == [0] * len(rects)
        for k, ref in enumerate(refs):
            assert np.array_equal(outs[k].cpu().numpy(), ref), "tile %d, repetition %d" % (k, rep)
    sc.close()
