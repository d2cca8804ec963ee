"""Host logic of bench.py (no GPU): the fixed CPU reference sample and the
reference arm's JSON line."""
import io
import json
import os
import sys
from contextlib import redirect_stdout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_cpu_tiles_cover_each_crop_once():
    for name, crop, spp, tile in bench.CPU_SAMPLE:
        x0, y0, x1, y1 = bench.cpu_crop(crop)
        assert x1 - x0 == crop and y1 - y0 == crop and 0 <= x0 and x1 <= bench.CPU_FRAME
        seen = set()
        for (a, b, c, d) in bench.cpu_tiles(crop, tile):
            assert x0 <= a < c <= x1 and y0 <= b < d <= y1
            for y in range(b, d):
                for x in range(a, c):
                    assert (x, y) not in seen
                    seen.add((x, y))
        assert len(seen) == crop * crop
        # enough tiles to spread over the host threads of a GPU box
        assert len(bench.cpu_tiles(crop, tile)) >= 16


def test_sample_covers_every_stream_scene():
    from xtracer_b200 import scenes
    assert sorted(n for n, *_ in bench.CPU_SAMPLE) == sorted(n for n, _ in scenes.JOBSTREAM_SCENES)
    assert sorted(bench.NCU_EXTEND) == sorted(n for n, _ in scenes.JOBSTREAM_SCENES)


class _Args:
    impl = "reference"
    gpus = 1
    steps = 2
    warmup = 1
    scale = 1.0


def _fake_runs(scale, threads, repeats):
    return [{"scene": n, "load_s": 0.5, "threads": threads,
             "renders": [{"render_s": 0.25 * (k + 1), "rays": 1000 * (k + 1)} for k in range(repeats)]}
            for n, *_ in bench.CPU_SAMPLE]


def test_reference_arm_line(monkeypatch):
    """The reference arm times the same sample as the cpu_baseline leg: step k
    is every scene's k-th render after the warm-up ones; value, e2e and
    cpu_baseline carry the same figure; no bytes cross to a GPU."""
    monkeypatch.setattr(bench, "cpu_reference_runs", _fake_runs)
    monkeypatch.setattr(bench, "dist_env", lambda: (0, 1, 0))
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.reference_arm(_Args()) == 0
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    n = len(bench.CPU_SAMPLE)
    rays = n * (2000 + 3000)
    secs = n * (0.5 + 0.75)
    assert line["impl"] == "reference" and line["unit"] == "Mrays/s" and line["higher_is_better"]
    assert abs(line["value"] - rays / secs / 1e6) < 1e-12
    assert line["e2e"] == {"value": line["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"
    assert line["cpu_baseline"]["sample"] == line["config"]["sample"] == bench.cpu_sample_text()
    assert set(line["cpu_baseline"]["per_scene"]) == {n for n, *_ in bench.CPU_SAMPLE}


def test_reference_arm_unavailable(monkeypatch):
    monkeypatch.setattr(bench, "cpu_reference_runs", lambda *a: None)
    monkeypatch.setattr(bench, "dist_env", lambda: (0, 1, 0))
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.reference_arm(_Args()) == 0
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_other_ranks_print_nothing(monkeypatch):
    monkeypatch.setattr(bench, "dist_env", lambda: (1, 2, 1))
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.reference_arm(_Args()) == 0
    assert buf.getvalue() == ""
