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
