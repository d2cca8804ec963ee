"""Render service on the GPU: a job's frame is the same alone and in the mix,
whatever the wave size, merging and graph replay; admission respects the
memory budget; latency bookkeeping is consistent."""
import ctypes as C

import numpy as np
import pytest

from xtracer_b200 import scenes, xtgpu
from xtracer_b200.service import Service

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    xtgpu.lib()
    yield


@pytest.fixture(scope="module")
def resident():
    fm = (xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8)
    return [xtgpu.Scene(scenes.spheres_scene(64, seed=1, name="s64"), node_formats=fm),
            xtgpu.Scene(scenes.terrain_scene(20_000, seed=2, name="t20k"), node_formats=fm),
            xtgpu.Scene(scenes.hairball_scene(20_000, seed=3, name="h20k"), node_formats=fm)]


JOBS = [(0, xtgpu.PATHTRACER, 64, 48, 8, 4, 100.0, 11), (1, xtgpu.PATHTRACER, 40, 40, 16, 4, 100.0, 12),
        (2, xtgpu.AO, 32, 32, 8, 4, 0.2, 13), (1, xtgpu.DEPTH, 50, 30, 2, 1, 100.0, 14),
        (0, xtgpu.STENCIL, 33, 17, 3, 1, 100.0, 15), (2, xtgpu.PATHTRACER, 24, 24, 4, 4, 100.0, 16)]


@pytest.mark.parametrize("fmt", [xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8])
def test_job_alone_equals_job_in_mix(resident, fmt):
    alone = []
    for (s, integ, w, h, spp, d, md, seed) in JOBS:
        img, _ = resident[s].render(integ, w, h, spp=spp, rdepth=d, ao_max_distance=md, seed=seed, node_format=fmt)
        alone.append(img)
    # small waves split every job over many waves; with two in flight their
    # accumulates overlap other waves' kernels and must still fold in order
    for wave, graphs, inflight in ((1 << 22, True, 2), (777, True, 2), (777, True, 1), (5000, False, 2),
                                   (777, True, 3), (901, True, 4)):
        svc = Service(resident, node_format=fmt, wave_paths=wave, use_graphs=graphs, merge_jobs=True,
                      memory_budget=1 << 30, waves_in_flight=inflight)
        ids = [svc.submit(s, integ, w, h, spp, d, md, seed) for (s, integ, w, h, spp, d, md, seed) in JOBS]
        svc.run()
        for jid, ref in zip(ids, alone):
            st = svc.poll(jid)
            assert st.state == 2
            out = svc.result(jid)
            assert np.array_equal(out, ref), "job %d differs in the mix (wave=%d)" % (jid, wave)
            svc.release(jid)
        svc.close()


def test_plain_path_equals_served(resident):
    plain = Service(resident, node_format=xtgpu.NODES_FP32, use_graphs=False, merge_jobs=False)
    served = Service(resident, node_format=xtgpu.NODES_FP32, use_graphs=True, merge_jobs=True)
    a = [plain.submit(*j) for j in JOBS]
    b = [served.submit(*j) for j in JOBS]
    plain.run()
    served.run()
    for x, y in zip(a, b):
        assert np.array_equal(plain.result(x), served.result(y))
        assert plain.poll(x).rays == served.poll(y).rays
    plain.close()
    served.close()


def test_memory_budget_limits_concurrency(resident):
    # budget for exactly one 64x64 frame: jobs run one after another
    svc = Service(resident, memory_budget=64 * 64 * 16, merge_jobs=True, host_results=True)
    ids = [svc.submit(0, xtgpu.STENCIL, 64, 64, 1, 1, 100.0, k) for k in range(4)]
    big = svc.submit(0, xtgpu.STENCIL, 128, 128, 1, 1, 100.0, 9)   # never fits
    svc.run()
    sts = [svc.poll(i) for i in ids]
    assert all(s.state == 2 for s in sts)
    for s0, s1 in zip(sts, sts[1:]):
        # admitted once the previous frame's device memory is freed (behind
        # its host copy, which may land later)
        assert s1.start_s >= s0.render_done_s - 1e-6
        assert s0.finish_s >= s0.render_done_s
    assert svc.poll(big).state == 3
    svc.close()


@pytest.mark.parametrize("inflight", [1, 2, 4])
def test_host_results_match(resident, inflight):
    """host_results: frames copied to pinned host memory asynchronously (device
    frames freed behind the copies) equal the frames of a plain render; the
    zero-copy view and the copy agree; pinned buffers are reused after release."""
    alone = [resident[s].render(integ, w, h, spp=spp, rdepth=d, ao_max_distance=md, seed=seed)[0]
             for (s, integ, w, h, spp, d, md, seed) in JOBS]
    svc = Service(resident, wave_paths=3000, merge_jobs=True, host_results=True, waves_in_flight=inflight)
    for rep in range(2):
        ids = [svc.submit(*j) for j in JOBS]
        svc.run()
        for jid, ref in zip(ids, alone):
            assert svc.poll(jid).state == 2
            view = svc.result_view(jid)
            assert np.array_equal(view, ref)
            assert np.array_equal(svc.result(jid), ref)
            svc.release(jid)
    svc.close()


def test_host_results_many_frames_of_one_class(resident):
    """40 finished 64x64 frames held at once: pinned frames of one size class
    are carved 16 to a pinned chunk, so this takes three chunks; every frame
    keeps its own buffer and equals its plain render (distinct seeds, so two
    jobs sharing a buffer would show), and the buffers are reused afterwards."""
    jobs = [(k % len(resident), xtgpu.PATHTRACER, 64, 64, 1, 2, 100.0, 100 + k) for k in range(40)]
    alone = [resident[s].render(integ, w, h, spp=spp, rdepth=d, ao_max_distance=md, seed=seed)[0]
             for (s, integ, w, h, spp, d, md, seed) in jobs]
    svc = Service(resident, merge_jobs=True, host_results=True)
    for rep in range(2):
        ids = [svc.submit(*j) for j in jobs]
        svc.run()
        for jid, ref in zip(ids, alone):
            assert svc.poll(jid).state == 2
            assert np.array_equal(svc.result_view(jid), ref)
        assert len({svc.result_view(jid).ctypes.data for jid in ids}) == len(ids)
        for jid in ids:
            svc.release(jid)
    svc.close()


def test_arrivals_and_latency_bookkeeping(resident):
    svc = Service(resident, merge_jobs=True)
    ids = [svc.submit(0, xtgpu.PATHTRACER, 32, 32, 4, 4, 100.0, k, submit_s=0.05 * k) for k in range(5)]
    svc.run()
    for k, i in enumerate(ids):
        st = svc.poll(i)
        assert st.state == 2
        assert st.submit_s == pytest.approx(0.05 * k)
        assert st.start_s >= st.submit_s - 1e-6
        assert st.finish_s >= st.render_done_s >= st.start_s
        assert st.rays > 0
    svc.close()


def test_autotune_keeps_results(resident):
    """The autotuner changes leaf size, stack, tile, register cap and wave size,
    never the result: depth and stencil frames are the same before and after."""
    from xtracer_b200 import scenes as sc_mod
    s = xtgpu.Scene(sc_mod.terrain_scene(50_000, seed=21, name="tune"))
    before = [s.render(k, 96, 64, spp=2)[0] for k in (xtgpu.STENCIL, xtgpu.DEPTH)]
    t = s.autotune(xtgpu.NODES_FP32, budget_ms=5000)
    assert t.leaf_size in (1, 2, 4) and t.tile in (0, 4, 8, 16) and t.extend_min_blocks in (0, 8, 10)
    assert t.stack_entries in (0, 32, 64) and t.wave_paths in (1 << 20, 1 << 22)
    got = s.tuning()
    assert (got.leaf_size, got.tile, got.wave_paths) == (t.leaf_size, t.tile, t.wave_paths)
    after = [s.render(k, 96, 64, spp=2)[0] for k in (xtgpu.STENCIL, xtgpu.DEPTH)]
    assert np.array_equal(before[0], after[0])
    assert np.array_equal(before[1], after[1])
    s.close()


def test_scene_tuning_reports_the_built_tree(resident):
    """A scene that was never tuned reports the process-wide tuning with its
    own leaf size and builder, so a read-modify-write of its tuning is
    accepted and changes nothing it renders."""
    sc = resident[0]
    t = sc.tuning()
    assert t.leaf_size == 2 and t.bvh_builder == 0   # Scene() builds leaves of 2 with LBVH
    ref, _ = sc.render(xtgpu.PATHTRACER, 32, 24, spp=2, rdepth=4, seed=3, node_format=xtgpu.NODES_W8)
    keep = {k: getattr(t, k) for k, _ in xtgpu.Tuning._fields_}
    try:
        sc.set_tuning(primary_variant=0)
        got, _ = sc.render(xtgpu.PATHTRACER, 32, 24, spp=2, rdepth=4, seed=3, node_format=xtgpu.NODES_W8)
    finally:
        sc.set_tuning(**keep)
    assert np.array_equal(ref, got)


def test_live_submissions_join_waves_in_flight(resident):
    """Continuous batching with live arrivals: while one thread serves
    (xtgpu_service_run on an open service, GIL released), another submits jobs
    as waves of a long job are on the GPU.  They are admitted before that job
    finishes, so their paths share its waves, and each renders the same bits
    as alone; the run returns once the service is closed and drained."""
    import threading
    import time
    fmt = xtgpu.NODES_W8
    long_job = (1, xtgpu.PATHTRACER, 512, 512, 32, 4, 100.0, 21)   # 8 Mi paths: 256 waves of 2^15
    later = [(0, xtgpu.PATHTRACER, 64, 48, 8, 4, 100.0, 22), (2, xtgpu.AO, 48, 48, 8, 2, 0.2, 23),
             (1, xtgpu.DEPTH, 40, 30, 2, 1, 100.0, 24), (0, xtgpu.PATHTRACER, 96, 64, 4, 4, 100.0, 25),
             (2, xtgpu.PATHTRACER, 32, 32, 16, 4, 100.0, 26), (1, xtgpu.STENCIL, 33, 17, 3, 1, 100.0, 27)]
    alone = [resident[s].render(integ, w, h, spp=spp, rdepth=d, ao_max_distance=md, seed=seed, node_format=fmt)[0]
             for (s, integ, w, h, spp, d, md, seed) in [long_job] + later]
    svc = Service(resident, node_format=fmt, wave_paths=1 << 15, use_graphs=True, merge_jobs=True,
                  memory_budget=1 << 30, waves_in_flight=3)
    svc.open(True)
    errors = []

    def serve():
        try:
            svc.run(max_seconds=120.0)
        except Exception as e:   # reported on the main thread
            errors.append(e)

    th = threading.Thread(target=serve)
    th.start()
    j0 = svc.submit(*long_job)
    t = time.time()
    while svc.poll(j0).state != 1 and time.time() - t < 30:
        time.sleep(0.0005)
    ids = []
    for j in later:
        ids.append(svc.submit(*j))
        time.sleep(0.002)
    svc.open(False)
    th.join(timeout=120)
    assert not th.is_alive() and not errors, errors
    s0 = svc.poll(j0)
    assert s0.state == 2
    starts = [svc.poll(i).start_s for i in ids]
    print("[live] long job done at %.3fs; later jobs admitted at %s" % (s0.render_done_s, np.round(starts, 3)))
    assert sum(s < s0.render_done_s for s in starts) >= 3, (starts, s0.render_done_s)
    for jid, ref in zip([j0] + ids, alone):
        st = svc.poll(jid)
        assert st.state == 2 and st.start_s >= st.submit_s - 1e-6
        assert np.array_equal(svc.result(jid), ref), "job %d" % jid
        svc.release(jid)
    svc.close()


def test_run_while_running_is_refused(resident):
    """One thread at a time runs the service."""
    import threading
    import time
    svc = Service(resident, node_format=xtgpu.NODES_W8, merge_jobs=True)
    svc.open(True)
    th = threading.Thread(target=lambda: svc.run(max_seconds=30.0))
    th.start()
    time.sleep(0.2)
    with pytest.raises(xtgpu.XtgpuError) as e:
        svc.run()
    assert e.value.status == 7   # XTGPU_ERR_STATE
    svc.open(False)
    th.join(timeout=60)
    assert not th.is_alive()
    svc.close()


def test_live_submission_over_budget_fails_alone(resident):
    """A job whose frame can never fit the memory budget is marked failed when
    it reaches the head of the queue; the jobs submitted around it, live, still
    render to the same bits as alone."""
    import threading
    fmt = xtgpu.NODES_W8
    ok_jobs = [(0, xtgpu.PATHTRACER, 64, 48, 4, 4, 100.0, 31), (1, xtgpu.DEPTH, 40, 30, 2, 1, 100.0, 32)]
    alone = [resident[s].render(integ, w, h, spp=spp, rdepth=d, ao_max_distance=md, seed=seed, node_format=fmt)[0]
             for (s, integ, w, h, spp, d, md, seed) in ok_jobs]
    # a 1024 x 1024 frame is 16 MiB; the budget holds 4 MiB
    svc = Service(resident, node_format=fmt, wave_paths=1 << 15, merge_jobs=True, memory_budget=4 << 20)
    svc.open(True)
    th = threading.Thread(target=lambda: svc.run(max_seconds=60.0))
    th.start()
    a = svc.submit(*ok_jobs[0])
    big = svc.submit(0, xtgpu.PATHTRACER, 1024, 1024, 1, 4, 100.0, 33)
    b = svc.submit(*ok_jobs[1])
    svc.open(False)
    th.join(timeout=60)
    assert not th.is_alive()
    assert svc.poll(big).state == 3
    for jid, ref in zip((a, b), alone):
        assert svc.poll(jid).state == 2
        assert np.array_equal(svc.result(jid), ref)
        svc.release(jid)
    svc.close()
