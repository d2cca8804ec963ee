"""Python handle on the render service of libxtgpu.so (xtgpu_service_* in
include/xtgpu.h): resident scenes, memory-budget admission, merged wavefront
launches replayed as CUDA graphs, per-job latency."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import xtgpu
from .xtgpu import check, lib


class Service:
    def __init__(self, scenes, node_format: int = xtgpu.NODES_FP32, wave_paths: int = 0, use_graphs: bool = True,
                 merge_jobs: bool = True, memory_budget: int = 48 << 30, max_jobs: int = 512,
                 host_results: bool = False, time_kernels: bool = False, count_visits: bool = False,
                 policy: int = 0, waves_in_flight: int = 2, stream=None):
        o = xtgpu.ServiceOpts(memory_budget, max_jobs, wave_paths, node_format, int(use_graphs), int(merge_jobs),
                              int(host_results), int(time_kernels), int(count_visits), policy, waves_in_flight)
        h = C.c_void_p()
        check(lib().xtgpu_service_create(C.byref(o), xtgpu.stream_handle(stream), C.byref(h)))
        self.handle = h
        self.scene_ids = []
        self.shapes = {}
        for sc in scenes:
            sid = C.c_int32()
            check(lib().xtgpu_service_add_scene(self.handle, sc.handle, C.byref(sid)))
            self.scene_ids.append(sid.value)

    def update_scene(self, scene: int) -> None:
        """Takes a resident scene's tables again after Scene.update."""
        check(lib().xtgpu_service_update_scene(self.handle, self.scene_ids[scene]))

    def submit(self, scene: int, integrator: int, width: int, height: int, spp: int, rdepth: int = 4,
               ao_max_distance: float = 100.0, seed: int = 1, submit_s: float = -1.0, aa: int = 1,
               distribution: int = xtgpu.SAMPLES_GRID) -> int:
        d = xtgpu.JobDesc(self.scene_ids[scene], integrator, width, height, spp, rdepth, ao_max_distance, seed,
                          aa, distribution)
        jid = C.c_int64()
        check(lib().xtgpu_service_submit(self.handle, C.byref(d), submit_s, C.byref(jid)))
        self.shapes[jid.value] = (height, width)
        return jid.value

    def run(self, max_seconds: float = 0.0) -> None:
        """Serves until the submitted jobs are done (xtgpu_service_run).  The
        call releases the GIL, so other Python threads may submit, poll and
        release meanwhile; while the service is open it waits for them."""
        check(lib().xtgpu_service_run(self.handle, max_seconds))

    def open(self, on: bool = True) -> None:
        """Opens (or closes) the service to live submissions: an open service's
        run() waits for new jobs instead of returning when idle."""
        check(lib().xtgpu_service_open(self.handle, int(on)))

    def poll(self, jid: int) -> xtgpu.JobStatus:
        st = xtgpu.JobStatus()
        check(lib().xtgpu_service_poll(self.handle, jid, C.byref(st)))
        return st

    def result(self, jid: int, out: np.ndarray = None) -> np.ndarray:
        h, w = self.shapes[jid]
        if out is None:
            out = np.zeros((h, w, 4), np.float32)
        check(lib().xtgpu_service_result(self.handle, jid, out.ctypes.data_as(C.c_void_p)))
        return out

    def result_view(self, jid: int) -> np.ndarray:
        """The finished frame in the service's pinned host memory (host_results
        services), as a read-only array without a copy; valid until release."""
        h, w = self.shapes[jid]
        p = C.POINTER(C.c_float)()
        check(lib().xtgpu_service_result_host(self.handle, jid, C.byref(p)))
        a = np.ctypeslib.as_array(p, shape=(h, w, 4))
        a.flags.writeable = False
        return a

    def release(self, jid: int) -> None:
        check(lib().xtgpu_service_release(self.handle, jid))

    def stats(self) -> xtgpu.ServiceStats:
        st = xtgpu.ServiceStats()
        check(lib().xtgpu_service_get_stats(self.handle, C.byref(st)))
        return st

    def reset_stats(self) -> None:
        check(lib().xtgpu_service_reset_stats(self.handle))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().xtgpu_service_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
