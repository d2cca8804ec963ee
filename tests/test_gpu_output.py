"""xtgpu.save_png / save_exr: the GPU quantiser (xtgpu_frame_rgba8) applies
XTracer's PNG arithmetic (lib/nimg/img.cc:150-172: channel * 255, clamped at
255, truncated) to a frame on the device or on the host."""
import numpy as np
import pytest

from xtracer_b200 import xtgpu
from tests import xtcore_host as xh

pytestmark = pytest.mark.gpu


def _expected(frame):
    s = frame.astype(np.float32) * np.float32(255.0)
    s = np.where(np.isnan(s) | (s <= 0), 0, np.minimum(s, 255.0))
    return s.astype(np.uint8)


def test_save_png_from_device_and_host(tmp_path):
    import torch
    from PIL import Image
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    rng = np.random.default_rng(3)
    frame = (rng.random((37, 53, 4)) * 1.4).astype(np.float32)
    frame[5, 7, 1] = np.nan
    frame[6, 8] = [0.0, 1.0, 255.0 / 255.0, 0.999]
    want = _expected(frame)
    xtgpu.save_png(str(tmp_path / "host.png"), frame)
    xtgpu.save_png(str(tmp_path / "dev.png"), torch.from_numpy(frame).cuda())
    for name in ("host.png", "dev.png"):
        got = np.asarray(Image.open(tmp_path / name).convert("RGBA"))
        assert np.array_equal(got, want), name
    xtgpu.save_exr(str(tmp_path / "f.exr"), frame)
    e = xh.read_exr(str(tmp_path / "f.exr"))
    for k, c in enumerate("RGB"):
        assert np.array_equal(e[c], frame[..., k], equal_nan=True)
