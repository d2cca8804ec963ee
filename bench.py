#!/usr/bin/env python
"""Benchmark of the B200 ray-intersection / integrator backend on the served
job stream: 8 resident scenes (terrain 10k..1M triangles, a 2M-triangle
hairball, 64 and 4096 spheres), 512 seeded jobs with resolution in
{128,256,512,1024}^2, spp in {1,4,16,64}, pathtracer depth 4.

A step is one slice of 64 jobs of that stream, all submitted at once and run
to completion through the render service (merged waves, three in flight, 8-bit
quantised BVH, CUDA graphs).  Reported beside it, on the same jobs: the plain path (one job per
launch, FP32 BVH, no graphs), an end-to-end pass with every frame copied back
to host memory, open-loop p50/p99 latency under Poisson arrivals, the extend
kernel's roofline and the reference CPU renderer on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python -m torch.distributed.run --nproc-per-node N ... bench.py --gpus N
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("jobstream-512: 8 resident scenes (terrain 10k/50k/200k/500k/1M tris, hairball 2M tris, "
            "64 and 4096 spheres), jobs res {128,256,512,1024}^2 x spp {1,4,16,64}, pathtracer depth 4")
METRIC = ("Mrays/s of the served job stream (merged waves, 8-wide BVH with 8-bit quantised child bounds, "
          "CUDA graphs); p50/p99 job latency")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xtgpu", choices=["xtgpu", "reference"])
    ap.add_argument("--jobs-per-step", type=int, default=64)
    ap.add_argument("--scale", type=float, default=1.0, help="scene size scale (1.0 = the workload)")
    ap.add_argument("--stream-jobs", type=int, default=512)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-latency", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    return ap.parse_args()


def dist_env():
    from xtracer_b200 import replicas
    return replicas.env()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
SERVED_FORMAT = 2   # xtgpu.NODES_W8: 8-wide BVH, 8-bit quantised child bounds
WAVES_IN_FLIGHT = 3   # served form: waves on streams of their own, each filling the earlier ones' tails
# The served extend kernel (k_extend_pool<W8>) per scene, from one ncu capture
# each of 1,048,576 first-bounce rays (python -m xtracer_b200.profile_extend
# --scene <scene> --fmt w8 --rays 1048576 --iters 1): DRAM and L2 bytes per ray,
# the share of issue slots used, and active lanes per warp instruction.  The
# roofline's traffic is the DRAM figure of each scene times that scene's rays,
# per launch; the issue figures name the resource that binds the kernel.
NCU_EXTEND = {
    "terrain10k": (37, 482, 0.736, 12.2), "terrain50k": (41, 709, 0.739, 11.3),
    "terrain200k": (50, 892, 0.731, 11.0), "terrain500k": (65, 990, 0.724, 11.4),
    "terrain1m": (90, 1254, 0.712, 10.9), "hairball2m": (91, 1760, 0.688, 12.9),
    "spheres64": (34, 111, 0.638, 16.3), "spheres4096": (35, 153, 0.598, 16.3)}


def build_scenes(scale, autotune=False):
    """The resident scenes with FP32, Q8 and W8 nodes; with autotune, each
    scene's BVH builder (LBVH or PLOC), leaf size, extend kernel, stack, tile,
    register cap and wave size are picked by xtgpu_autotune for the served
    format (W8)."""
    from xtracer_b200 import scenes, xtgpu
    out, specs, tunes = [], [], {}
    for name, _ in scenes.JOBSTREAM_SCENES:
        spec = scenes.jobstream_scene(name, scale)
        specs.append(spec)
        sc = xtgpu.Scene(spec, node_formats=(xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8), leaf_size=1)
        if autotune:
            t = sc.autotune(SERVED_FORMAT, budget_ms=2000)
            for f in (xtgpu.NODES_FP32, xtgpu.NODES_Q8, xtgpu.NODES_W8):
                sc.build_bvh(f, t.leaf_size)
            tunes[name] = {k: getattr(t, k) for k in ("leaf_size", "extend_variant", "steps_per_vote",
                                                       "primary_node_format", "primary_variant", "stack_entries",
                                                       "tile", "extend_min_blocks", "wave_paths", "bvh_builder")}
        out.append(sc)
    return specs, out, tunes


def run_slice(svc, jobs, record=None, per_scene=None, view=False, job_stats=None):
    """Submits the jobs at once, runs the service to completion; returns
    (rays, latencies in s).  per_scene (array) accumulates rays by scene.
    record collects each frame (copied), or with view (host_results services)
    the last pixel read from the frame's host copy in place.  job_stats, a
    pair of lists, collects each job's rays and its time from admission to
    its last wave."""
    from xtracer_b200 import xtgpu
    ids = [svc.submit(j.scene, xtgpu.PATHTRACER, j.width, j.height, j.spp, j.depth, 100.0, j.seed) for j in jobs]
    svc.run()
    rays, lat = 0, []
    for j, i in zip(jobs, ids):
        st = svc.poll(i)
        if st.state != 2:
            raise RuntimeError("job %d did not finish (state %d)" % (i, st.state))
        rays += st.rays
        if per_scene is not None:
            per_scene[j.scene] += st.rays
        lat.append(st.finish_s - st.submit_s)
        if job_stats is not None:
            job_stats[0].append(st.rays)
            job_stats[1].append(st.render_done_s - st.start_s)
        if record is not None:
            record.append(float(svc.result_view(i)[-1, -1, 0]) if view else svc.result(i))
        svc.release(i)
    return rays, lat


def serve_open_loop(svc, jobs, arrivals):
    """Open-loop serving with live arrivals: one thread runs the (open)
    service while this one submits each job when its arrival time (seconds
    from the start) comes, whatever is on the GPU then.  Returns the jobs'
    latencies (result available minus submission, service clock), their rays
    and the wall time from the first arrival to the last result."""
    from xtracer_b200 import xtgpu
    errors = []

    def serve():
        try:
            svc.run()
        except Exception as e:   # re-raised below
            errors.append(e)

    svc.open(True)
    th = threading.Thread(target=serve)
    th.start()
    ids = []
    t0 = time.perf_counter()
    for j, a in zip(jobs, arrivals):
        dt = float(a) - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        ids.append(svc.submit(j.scene, xtgpu.PATHTRACER, j.width, j.height, j.spp, j.depth, 100.0, j.seed))
    svc.open(False)
    th.join()
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0]
    lats, rays = [], 0
    for i in ids:
        st = svc.poll(i)
        if st.state != 2:
            raise RuntimeError("job %d did not finish (state %d)" % (i, st.state))
        lats.append(st.finish_s - st.submit_s)
        rays += st.rays
        svc.release(i)
    return lats, rays, wall


def full_wave_rates(services, specs):
    """Mrays/s of every scene when one job fills the GPU: a 1024x1024 x 16 spp
    pathtracer job (16 Mi paths, four full waves, depth 4) submitted alone to
    each service ({"plain": ..., "served": ...}); CUDA events around the
    service run, best of 3 after a warm-up."""
    import torch
    from xtracer_b200 import scenes
    out = {}
    for k, sp in enumerate(specs):
        row = {}
        job = [scenes.Job(0, k, 1024, 1024, 16, 4, 0.0, 99)]
        for tag, svc in services.items():
            best = None
            for it in range(4):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                rays, _ = run_slice(svc, job)
                e1.record()
                torch.cuda.synchronize()
                if it:
                    t = e0.elapsed_time(e1) / 1000.0
                    best = t if best is None else min(best, t)
            row[tag] = rays / best / 1e6
        out[sp.name] = row
    return out


def pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def roofline_bytes_per_ray(specs, gpu_scenes, node_format):
    """Algorithmic bytes per ray of the extend kernel, per scene:
    32 (ray) + 16 (hit) + nodes_visited * node_bytes + prims_tested * 48, with
    the visit counts measured once per scene by a counting traversal over a
    pathtracer job of that scene (128^2 x 4 spp, depth 4)."""
    from xtracer_b200 import xtgpu
    from xtracer_b200.service import Service
    node_bytes = xtgpu.NODE_BYTES[node_format]
    out = []
    for k, sc in enumerate(gpu_scenes):
        svc = Service(gpu_scenes, node_format=node_format, count_visits=True)
        jid = svc.submit(k, xtgpu.PATHTRACER, 128, 128, 4, 4, 100.0, 12345)
        svc.run()
        st = svc.stats()
        svc.release(jid)
        svc.close()
        vn = st.node_visits / max(st.rays, 1)
        vp = st.prim_tests / max(st.rays, 1)
        out.append({"scene": specs[k].name, "nodes_per_ray": vn, "prims_per_ray": vp,
                    "bytes_per_ray": 32 + 16 + vn * node_bytes + vp * 48})
    return out


# ---------------------------------------------------------------------------
# The fixed sample the reference renderer (oracle/_ref/xtref: XTracer's xtcore
# built from its sources) is timed on, the same in the --impl reference arm and
# in the cpu_baseline leg: for each of the 8 resident scenes, one pathtracer
# job of the stream's kind (256x256 frame, depth 4, seed 7) rendered on a
# centred crop.  Crop edge and spp per scene keep each render to a few seconds
# on the host cores; the reference's cost per ray grows with the mesh
# (Octree::r_intersection tests every triangle of every node a ray's box
# meets, octree.tml:206-249).  The reference renders tiles in parallel
# (integrator.cc:40-42), so each crop is handed over as tiles of the given edge,
# enough of them for every host thread.  Scene load and octree build are timed
# apart.
CPU_SAMPLE = [("terrain10k", 32, 4, 2), ("terrain50k", 20, 4, 2), ("terrain200k", 12, 4, 1),
              ("terrain500k", 8, 4, 1), ("terrain1m", 6, 4, 1), ("hairball2m", 6, 1, 1), ("spheres64", 64, 16, 4),
              ("spheres4096", 24, 4, 2)]
CPU_FRAME = 256


def cpu_sample_text():
    return ("pathtracer depth 4, seed 7, on centred crops of %dx%d frames in tiles: " % (CPU_FRAME, CPU_FRAME) +
            ", ".join("%s %dx%d x %d spp (%dx%d tiles)" % (n, c, c, spp, t, t) for n, c, spp, t in CPU_SAMPLE) +
            " (IIntegrator::render timed, rays counted at Scene::intersection; scene load and octree build "
            "timed apart)")


def cpu_crop(c):
    x0 = (CPU_FRAME - c) // 2
    return (x0, x0, x0 + c, x0 + c)


def cpu_tiles(c, t):
    x0, y0, x1, y1 = cpu_crop(c)
    return [(x, y, min(x + t, x1), min(y + t, y1)) for y in range(y0, y1, t) for x in range(x0, x1, t)]


def cpu_reference_runs(scale, threads, repeats):
    """Per scene of CPU_SAMPLE: the reference loads the scene once and renders
    its crop `repeats` times.  Returns [{"scene", "load_s", "renders": [...]}]
    or None when the harness is not built."""
    from oracle import pyoracle as po
    from xtracer_b200 import scenes
    if not po.ref_available():
        return None
    work = tempfile.mkdtemp(prefix="xtref")
    out = []
    for name, crop, spp, tile in CPU_SAMPLE:
        spec = scenes.jobstream_scene(name, scale)
        scn = spec.write_scn(work)
        r = po.ref_bench(scn, "pathtracer", CPU_FRAME, CPU_FRAME, spp, 4, threads, 7, cpu_tiles(crop, tile), repeats,
                         workdir=work)
        r["scene"] = name
        out.append(r)
    return out


def cpu_reference_sample(scale, threads):
    """The cpu_baseline leg: one untimed and one timed render of every crop of
    the sample; Mrays/s over the timed renders, per scene and in total."""
    runs = cpu_reference_runs(scale, threads, 2)
    if runs is None:
        return None
    rays = sum(r["renders"][1]["rays"] for r in runs)
    secs = sum(r["renders"][1]["render_s"] for r in runs)
    return {"value": rays / secs / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": cpu_sample_text(), "rays": rays, "seconds": secs,
            "per_scene": {r["scene"]: {"mrays": r["renders"][1]["rays"] / r["renders"][1]["render_s"] / 1e6,
                                       "rays": r["renders"][1]["rays"], "render_s": r["renders"][1]["render_s"],
                                       "load_s": r["load_s"]} for r in runs}}


def gpu_on_cpu_sample(gscenes, specs):
    """The GPU (xtgpu_render, FP32 nodes, one job per call) on the jobs of the
    CPU sample: each crop as the CPU rendered it, and the job's whole frame;
    Mrays/s per scene from CUDA events (best of 3 after a warm-up)."""
    import torch
    from xtracer_b200 import xtgpu
    names = [s.name for s in specs]
    out = {}
    for name, crop, spp, _ in CPU_SAMPLE:
        sc = gscenes[names.index(name)]
        row = {}
        for tag, rect in (("crop", cpu_crop(crop)), ("frame", None)):
            best = None
            for it in range(4):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                _, rays = sc.render(xtgpu.PATHTRACER, CPU_FRAME, CPU_FRAME, spp=spp, rdepth=4, seed=7, rect=rect)
                e1.record()
                torch.cuda.synchronize()
                if it:
                    t = e0.elapsed_time(e1) / 1000.0
                    best = t if best is None else min(best, t)
            row[tag + "_mrays"] = rays / best / 1e6
        out[name] = row
    return out


def reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    runs = cpu_reference_runs(args.scale, threads, args.warmup + args.steps)
    if runs is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/xtref was not built"}))
        return 0
    # step k: every crop of the sample rendered once (the k-th render of each
    # scene's process); the scenes were loaded before the first step
    steps = range(args.warmup, args.warmup + args.steps)
    t_all = sum(r["renders"][k]["render_s"] for r in runs for k in steps)
    r_all = sum(r["renders"][k]["rays"] for r in runs for k in steps)
    value = r_all / t_all / 1e6
    per_scene = {r["scene"]: {"mrays": sum(r["renders"][k]["rays"] for k in steps) /
                              sum(r["renders"][k]["render_s"] for k in steps) / 1e6,
                              "load_s": r["load_s"]} for r in runs}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_all / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded scenes and job stream)",
            "config": {"workload": WORKLOAD, "sample": cpu_sample_text()},
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                             "sample": cpu_sample_text(), "per_scene": per_scene},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    # the services launch on this stream and the step events are recorded on it
    # (the legacy default stream cannot be captured into CUDA graphs)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    from xtracer_b200 import replicas, scenes, xtgpu
    from xtracer_b200.service import Service
    D = replicas.Group(world, "nccl")

    specs, gscenes, tunes = build_scenes(args.scale, autotune=not args.no_autotune)
    jobs = replicas.rank_stream(rank, args.stream_jobs)
    nslices = max(1, len(jobs) // args.jobs_per_step)
    slices = [jobs[i * args.jobs_per_step:(i + 1) * args.jobs_per_step] for i in range(nslices)]
    budget = 48 << 30

    served = Service(gscenes, node_format=SERVED_FORMAT, use_graphs=True, merge_jobs=True, memory_budget=budget,
                     waves_in_flight=WAVES_IN_FLIGHT, stream=stream)
    # warm-up steps (untimed): graphs captured, allocator pools primed
    for w in range(args.warmup):
        run_slice(served, slices[w % nslices])
    served.reset_stats()
    timed = [slices[(args.warmup + k) % nslices] for k in range(args.steps)]

    clocks = ClockSampler(local)
    D.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rays, lat = 0, []
    for sl in timed:
        r, l = run_slice(served, sl)
        rays += r
        lat += l
    e1.record()
    torch.cuda.synchronize()
    D.barrier()
    clk = clocks.stop()
    dev_s = e0.elapsed_time(e1) / 1000.0
    st = served.stats()
    t_max = D.max(dev_s)
    rays_all = D.sum(rays)
    value = rays_all / t_max / 1e6
    lat_all = D.gather(lat)

    # roofline of the W8 extend kernel: the same steps again, one wave at a time
    # (with two waves in flight, an extend launch's CUDA-event span includes the
    # other wave's kernels), every pass on W8 nodes so that the timed launches
    # and the counted node visits are all of that kernel
    saved = [{k: getattr(sc.tuning(), k) for k, _ in xtgpu.Tuning._fields_} for sc in gscenes]
    for sc in gscenes:
        sc.set_tuning(primary_node_format=-1)
    rsvc = Service(gscenes, node_format=SERVED_FORMAT, use_graphs=True, merge_jobs=True, memory_budget=budget,
                   time_kernels=True, waves_in_flight=1, stream=stream)
    run_slice(rsvc, slices[0])
    rsvc.reset_stats()
    per_scene = np.zeros(len(gscenes))
    for sl in timed:
        run_slice(rsvc, sl, per_scene=per_scene)
    rst = rsvc.stats()
    rsvc.close()
    bpr = roofline_bytes_per_ray(specs, gscenes, SERVED_FORMAT)
    for sc, t in zip(gscenes, saved):
        sc.set_tuning(**t)
    scene_bpr = [b["bytes_per_ray"] for b in bpr]
    # rays of each scene in the timed steps times that scene's bytes per ray
    alg_bytes = float(np.dot(per_scene, scene_bpr))
    ext_s = rst.extend_ms / 1000.0
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / ext_s / 1e9 if ext_s > 0 else None
    rays_per_launch = float(per_scene.sum()) / max(1, rst.extend_launches)
    ncu_rows = [NCU_EXTEND[sp.name] for sp in specs]
    wsum = max(1.0, float(per_scene.sum()))
    wavg = lambda k: float(sum(per_scene[i] * ncu_rows[i][k] for i in range(len(specs)))) / wsum
    traffic = wavg(0) * rays_per_launch

    # end to end: same steps, every frame copied to host memory by the service
    e2e_svc = Service(gscenes, node_format=SERVED_FORMAT, use_graphs=True, merge_jobs=True, memory_budget=budget,
                      host_results=True, waves_in_flight=WAVES_IN_FLIGHT, stream=stream)
    # untimed warm-up: the served arm's warm-up steps, then each distinct step
    # of the timed region once, so that the pinned host pool holds as many
    # frames of each size class as a step needs (a steady-state server pins no
    # memory per job; pinning a cold pool costs about 14 % in its first pass)
    for w in range(args.warmup):
        run_slice(e2e_svc, slices[w % nslices], record=[], view=True)
    for k in sorted({(args.warmup + k) % nslices for k in range(args.steps)} - {w % nslices for w in range(args.warmup)}):
        run_slice(e2e_svc, slices[k], record=[], view=True)
    D.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_rays = 0
    d2h = 0
    for sl in timed:
        r, _ = run_slice(e2e_svc, sl, record=[], view=True)
        e_rays += r
        d2h += sum(j.width * j.height * 16 for j in sl)
    torch.cuda.synchronize()
    e2e_s = D.max(time.perf_counter() - t0)
    e2e_value = D.sum(e_rays) / e2e_s / 1e6
    e2e_svc.close()

    # plain path: one job per launch, FP32 BVH, no graphs, on the first timed step
    plain = None
    if not args.no_plain:
        psvc = Service(gscenes, node_format=xtgpu.NODES_FP32, use_graphs=False, merge_jobs=False,
                       memory_budget=budget, waves_in_flight=1, stream=stream)
        run_slice(psvc, slices[0])   # warm-up: allocator pools, modules
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        psvc_jobs, psvc_times = [], []
        p0.record()
        pr, pl = run_slice(psvc, timed[0], job_stats=(psvc_jobs, psvc_times))
        p1.record()
        torch.cuda.synchronize()
        ps = p0.elapsed_time(p1) / 1000.0
        # equal RMSE (untimed): frames of the step's first jobs from the plain
        # path and from the served form; every node format and kernel returns
        # the same hits, so the frames are equal bit for bit
        check_jobs = timed[0][:16]
        pf, sf = [], []
        run_slice(psvc, check_jobs, record=pf)
        run_slice(served, check_jobs, record=sf)
        diff = max(float(np.nanmax(np.abs(a - b))) if a.size else 0.0 for a, b in zip(pf, sf))
        same = all(np.array_equal(a, b, equal_nan=True) for a, b in zip(pf, sf))
        del pf, sf
        # the served path on exactly that step, for a like-for-like ratio
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        sr, sl_ = run_slice(served, timed[0])
        s1.record()
        torch.cuda.synchronize()
        ss = s0.elapsed_time(s1) / 1000.0
        # the served form with W8 nodes for the camera rays too (no binary pass)
        saved = [{k: getattr(sc.tuning(), k) for k, _ in xtgpu.Tuning._fields_} for sc in gscenes]
        for sc in gscenes:
            sc.set_tuning(primary_node_format=-1)
        run_slice(served, slices[0])   # captures the graphs of this tuning
        torch.cuda.synchronize()
        w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0.record()
        wr, _ = run_slice(served, timed[0])
        w1.record()
        torch.cuda.synchronize()
        w8_only = wr / (w0.elapsed_time(w1) / 1000.0) / 1e6
        for sc, t in zip(gscenes, saved):
            sc.set_tuning(**t)
        # the served form with the other node formats on that step
        other = {}
        for fname, f in (("fp32", xtgpu.NODES_FP32), ("q8", xtgpu.NODES_Q8)):
            fsvc = Service(gscenes, node_format=f, use_graphs=True, merge_jobs=True,
                           memory_budget=budget, waves_in_flight=WAVES_IN_FLIGHT, stream=stream)
            run_slice(fsvc, slices[0])
            torch.cuda.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record()
            fr, _ = run_slice(fsvc, timed[0])
            f1.record()
            torch.cuda.synchronize()
            other[fname] = fr / (f0.elapsed_time(f1) / 1000.0) / 1e6
            fsvc.close()
        # where the plain path's time goes: each job of the step at its scene's
        # full-wave rate would take rays / rate; the rest of its time is the
        # cost of a job too small to fill the GPU (short waves, launch tails,
        # per-job set-up).  That bounds what merging jobs can win, and the node
        # format what the faster traversal can.
        rates = full_wave_rates({"plain": psvc, "served": served}, specs)
        jids = psvc_jobs
        ideal_p = sum(r / (rates[specs[j.scene].name]["plain"] * 1e6) for j, r in zip(timed[0], jids))
        ideal_s = sum(r / (rates[specs[j.scene].name]["served"] * 1e6) for j, r in zip(timed[0], jids))
        small = [k for k, j in enumerate(timed[0]) if j.width * j.height * j.spp < (1 << 20)]
        breakdown = {"plain_s": ps, "served_s": ss,
                     "plain_at_full_wave_rate_s": ideal_p, "served_at_full_wave_rate_s": ideal_s,
                     "bound_merging_only": ps / ideal_p, "bound_merging_and_served_kernels": ps / ideal_s,
                     "achieved": ps / ss, "jobs_under_1Mi_paths": len(small),
                     "their_share_of_plain_s": sum(psvc_times[k] for k in small) / ps,
                     "their_share_of_rays": sum(jids[k] for k in small) / max(1, sum(jids)),
                     "full_wave_mrays": rates}
        psvc.close()
        plain = {"value": pr / ps / 1e6, "unit": "Mrays/s", "step_jobs": len(timed[0]), "breakdown": breakdown,
                 "p50_ms": 1000 * pct(pl, 50), "p99_ms": 1000 * pct(pl, 99),
                 "served_same_step_mrays": sr / ss / 1e6, "speedup": (sr / ss) / (pr / ps),
                 "served_w8_only_same_step_mrays": w8_only,
                 "served_fp32_same_step_mrays": other["fp32"], "served_q8_same_step_mrays": other["q8"],
                 "form": "one job per launch, FP32 BVH, no CUDA graphs",
                 "equal_rmse": {"jobs": len(check_jobs), "frames_bit_identical": bool(same),
                                "max_abs_diff": diff}}

    # open-loop latency over the rank's whole stream: its jobs arrive as a
    # Poisson process at 1.5x the plain path's job rate (offered load above the
    # plain path's capacity) and are submitted live while earlier jobs are on
    # the GPU; the served form and the plain path on the same arrivals
    latency = None
    if not args.no_latency:
        rate = 1.5 * len(timed[0]) / ps if plain is not None else 50.0
        arr = np.cumsum(np.random.default_rng(4 + rank).exponential(1.0 / rate, len(jobs)))
        arr -= arr[0]
        lsvc = Service(gscenes, node_format=SERVED_FORMAT, use_graphs=True, merge_jobs=True, memory_budget=budget,
                       waves_in_flight=WAVES_IN_FLIGHT, stream=stream)
        run_slice(lsvc, slices[0])   # graphs of this service captured before the arrivals start
        lats, lrays, lwall = serve_open_loop(lsvc, jobs, arr)
        lsvc.close()
        lat_all_open = D.gather(lats)
        # the same arrivals with waves shared equally between the running jobs
        # (policy 1) instead of fewest remaining paths first
        esvc = Service(gscenes, node_format=SERVED_FORMAT, use_graphs=True, merge_jobs=True, memory_budget=budget,
                       waves_in_flight=WAVES_IN_FLIGHT, stream=stream, policy=1)
        run_slice(esvc, slices[0])
        elats, erays, ewall = serve_open_loop(esvc, jobs, arr)
        esvc.close()
        elat_all = D.gather(elats)
        latency = {"arrivals": "Poisson, %.2f jobs/s (1.5x the plain path's job rate), submitted live" % rate,
                   "jobs": len(lat_all_open), "p50_ms": 1000 * pct(lat_all_open, 50),
                   "p99_ms": 1000 * pct(lat_all_open, 99), "max_ms": 1000 * max(lat_all_open),
                   "mrays_s_wall": D.sum(lrays) / D.max(lwall) / 1e6, "wall_s": D.max(lwall),
                   "memory_budget_gb": budget / 2 ** 30, "policy": "fewest remaining paths first",
                   "equal_share": {"p50_ms": 1000 * pct(elat_all, 50), "p99_ms": 1000 * pct(elat_all, 99),
                                   "max_ms": 1000 * max(elat_all), "wall_s": D.max(ewall),
                                   "mrays_s_wall": D.sum(erays) / D.max(ewall) / 1e6}}
        if plain is not None:
            psvc = Service(gscenes, node_format=xtgpu.NODES_FP32, use_graphs=False, merge_jobs=False,
                           memory_budget=budget, waves_in_flight=1, stream=stream)
            plats, prays, pwall = serve_open_loop(psvc, jobs, arr)
            plat_all = D.gather(plats)
            latency["plain"] = {"p50_ms": 1000 * pct(plat_all, 50), "p99_ms": 1000 * pct(plat_all, 99),
                                "max_ms": 1000 * max(plat_all), "wall_s": D.max(pwall),
                                "mrays_s_wall": D.sum(prays) / D.max(pwall) / 1e6}
            # both forms at an offered load the plain path can carry (0.8x its
            # job rate), where the percentiles are those of a stable queue
            arr8 = arr * (1.5 / 0.8)
            qsvc = Service(gscenes, node_format=SERVED_FORMAT, use_graphs=True, merge_jobs=True,
                           memory_budget=budget, waves_in_flight=WAVES_IN_FLIGHT, stream=stream)
            run_slice(qsvc, slices[0])
            q8, _, qw = serve_open_loop(qsvc, jobs, arr8)
            qsvc.close()
            p8, _, pw8 = serve_open_loop(psvc, jobs, arr8)
            psvc.close()
            q8, p8 = D.gather(q8), D.gather(p8)
            latency["at_0.8x_plain_rate"] = {
                "jobs_per_s": 0.8 * len(timed[0]) / ps,
                "served": {"p50_ms": 1000 * pct(q8, 50), "p99_ms": 1000 * pct(q8, 99), "wall_s": D.max(qw)},
                "plain": {"p50_ms": 1000 * pct(p8, 50), "p99_ms": 1000 * pct(p8, 99), "wall_s": D.max(pw8)}}

    # the reference on the host cores: rank 0 of a one-GPU run only (with
    # replicas, the host's cores are shared by the ranks' own host work)
    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_reference_sample(args.scale, os.cpu_count() or 1)
        if cpu is not None:
            gpu_same = gpu_on_cpu_sample(gscenes, specs)
            for name, row in gpu_same.items():
                cpu["per_scene"][name].update({"gpu_" + k: v for k, v in row.items()})
            # the reference's rate on the served stream's own ray mix: the CPU
            # time of each scene's rays in the timed steps at that scene's rate
            cpu_s = sum(per_scene[k] / (cpu["per_scene"][sp.name]["mrays"] * 1e6)
                        for k, sp in enumerate(specs) if per_scene[k] > 0)
            cpu["stream_mix_mrays"] = float(per_scene.sum()) / cpu_s / 1e6 if cpu_s > 0 else None
    served.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes and job stream)",
            "config": {"workload": WORKLOAD, "jobs_per_step": args.jobs_per_step, "scale": args.scale,
                       "parallelism": "replicas" if world > 1 else "single",
                       "cache": "inputs larger than L2 (resident scenes ~%.0f MB)" %
                                (sum(s.device_bytes() for s in gscenes) / 1e6),
                       "wave_paths": 1 << 22, "node_format": "w8 (8-wide, 8-bit quantised) for bounce rays; camera rays as tuned "
                                      "per scene (primary_node_format: 0 = binary FP32, -1 = w8)",
                       "cuda_graphs": True, "waves_in_flight": WAVES_IN_FLIGHT,
                       "autotuned": tunes},
            "p50_ms": 1000 * pct(lat_all, 50), "p99_ms": 1000 * pct(lat_all, 99),
            "latency_open_loop": latency, "plain": plain,
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": 64 * len(timed[0]),
                    "d2h_bytes_per_step": d2h // max(1, len(timed))},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "traffic_source": "ncu DRAM read+write of k_extend_pool<W8> per scene on 1 Mi "
                                           "first-bounce rays (%s B/ray), weighted by the timed steps' rays "
                                           "of each scene, times %.0f rays per launch" %
                                           ({sp.name: NCU_EXTEND[sp.name][0] for sp in specs}, rays_per_launch),
                         "binding": {"resource": "instruction issue: the kernel waits on dependent node "
                                                 "loads and runs a third of its lanes per instruction; DRAM "
                                                 "and L2 carry a small share of their bandwidth",
                                     "issue_active_frac": wavg(2), "simt_lanes_of_32": wavg(3),
                                     "l2_bytes_per_ray": wavg(1), "dram_bytes_per_ray": wavg(0),
                                     "source": "ncu per scene (profile_extend), weighted by the timed rays"},
                         "algorithmic_bytes_per_launch": alg_bytes / max(1, rst.extend_launches),
                         "kernel": "k_extend_pool<W8> / k_extend_batch<W8> (closest-hit traversal, 8-wide "
                                   "quantised nodes)", "peak_kind": peak_kind,
                         "extend_ms": rst.extend_ms, "extend_launches": rst.extend_launches,
                         "timing": "CUDA events around every extend launch, same steps, one wave in flight, "
                                   "all passes on W8 nodes",
                         "bytes_per_ray": {b["scene"]: round(b["bytes_per_ray"], 1) for b in bpr},
                         "nodes_per_ray": {b["scene"]: round(b["nodes_per_ray"], 2) for b in bpr},
                         "prims_per_ray": {b["scene"]: round(b["prims_per_ray"], 2) for b in bpr}},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(st.kernel_launches),
            "rays": rays_all,
        }
        print(json.dumps(line))
    D.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
