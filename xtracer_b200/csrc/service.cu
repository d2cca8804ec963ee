// Render service: resident scenes, memory-budget admission and merged
// wavefront launches.  No counterpart in the reference, whose renders are one
// blocking IIntegrator::render() call per frame (src/xtcore/integrator.cc:29-53).
//
// Each wave takes a share of the queue capacity from every admitted job
// (continuous batching): a job that arrives while others run joins the next
// wave as soon as a slot and memory for its frame are free.  A wave is one
// fixed kernel sequence (camera, [extend, shade] x bounces, accumulate) whose
// sizes live in device memory, so it replays as a CUDA graph.
//
// Two waves are in flight at a time, on two streams with their own queues:
// the next wave's camera, extend and shade kernels fill the SMs the previous
// wave's tail leaves idle, and its accumulate waits for the previous one.
//
// Because paths are keyed by (seed, pixel, sample) and folded per pixel in
// sample order, a job's frame is bit-identical whatever it is merged with.
//
// Threads: xtgpu_service_run runs the loop on the calling thread.  Other
// threads may submit, poll, read results, release jobs and open or close the
// service meanwhile: those calls and the loop's bookkeeping share one mutex,
// which the loop drops while it waits for a wave or for arrivals, and a
// submission wakes the loop.  A job submitted while waves are in flight is
// admitted as slots and memory free up and joins the next wave launched.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "render.h"

namespace xtg {

struct SvcJob {
    xtgpu_job_desc d{};
    int state = 0;   // 0 queued, 1 running, 2 done, 3 failed
    double submit_s = 0, start_s = 0, finish_s = 0, render_done_s = 0;
    int64_t paths = 0;
    int64_t planned = 0;   // paths given to launched waves
    int64_t done = 0;      // paths of retired waves
    uint64_t rays = 0;
    uint64_t frame_bytes = 0;
    float4 *frame = nullptr;
    float4 *host = nullptr;          // pinned host copy (host_results)
    uint64_t host_bytes = 0;         // its allocated size (a size class)
    cudaEvent_t copied = nullptr;    // set while the host copy is in flight
};

// Size class of a pinned host frame: the next power of two, at least 64 KB.
static uint64_t pinned_class(uint64_t bytes)
{
    uint64_t c = 1ull << 16;
    while (c < bytes) c <<= 1;
    return c;
}

// One wave in flight: its runner (queues, job table, graphs), the stream it
// runs on, and what the host needs when it retires.
struct WaveSlot {
    WaveRunner R;
    cudaStream_t s = nullptr;
    cudaEvent_t fin = nullptr;            // after the wave's accumulate and ray-count copy
    unsigned long long *jrays = nullptr;  // pinned: rays per job of the wave
    std::vector<DevJob> wave;
    std::vector<int64_t> ids;
};

}  // namespace xtg

struct xtgpu_service {
    xtgpu_service_opts o{};
    cudaStream_t s = nullptr;  // admission, frees, results
    bool own_stream = false;   // created here: the legacy default stream cannot be captured
    cudaStream_t cs = nullptr; // host_results: frame copies to pinned memory, off the
                               // admission stream that the next waves wait on
    int nslots = 2;
    xtg::WaveSlot slot[XTGPU_MAX_WAVES_IN_FLIGHT];
    cudaEvent_t admitted = nullptr;   // frames of admitted jobs allocated and zeroed
    std::vector<xtgpu_scene *> scenes;
    std::vector<xtg::DevScene> dev;
    std::map<int64_t, xtg::SvcJob> jobs;
    std::deque<int64_t> pending;     // submitted, not admitted (FIFO)
    std::vector<int64_t> active;     // admitted, not finished (admission order)
    int64_t next_id = 0;
    uint64_t mem_used = 0;
    std::chrono::steady_clock::time_point t0;
    uint64_t waves = 0;
    // host_results: pinned frames reused by size, events of copies in flight
    std::multimap<uint64_t, float4 *> pinned_free;
    std::vector<void *> pinned_chunks;   // what cudaMallocHost returned; frames are carved from these
    std::vector<cudaEvent_t> events_free;
    std::vector<int64_t> copying;    // finished on the GPU, host copy in flight
    // the job table and everything above it that submit, poll, result and
    // release touch; run() holds it except while it waits
    std::mutex mu;
    std::condition_variable arrived;  // a submission or xtgpu_service_open
    bool open = false;                // run() waits for submissions while set
    bool running = false;             // one run() at a time

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

using namespace xtg;

static xtgpu_status admit(xtgpu_service *v, double now)
{
    while (!v->pending.empty()) {
        int64_t id = v->pending.front();
        SvcJob &J = v->jobs[id];
        if (J.submit_s > now) break;
        int max_active = v->o.merge_jobs ? v->o.max_jobs : 1;
        if ((int)v->active.size() >= max_active) break;
        if (J.frame_bytes > v->o.memory_budget_bytes) {
            J.state = 3;   // can never fit
            v->pending.pop_front();
            continue;
        }
        if (v->mem_used + J.frame_bytes > v->o.memory_budget_bytes) break;
        XTG_CUDA(cudaMallocAsync((void **)&J.frame, J.frame_bytes, v->s));
        XTG_CUDA(cudaMemsetAsync(J.frame, 0, J.frame_bytes, v->s));
        v->mem_used += J.frame_bytes;
        J.state = 1;
        J.start_s = now;
        v->active.push_back(id);
        v->pending.pop_front();
    }
    return XTGPU_OK;
}

// Plans a wave over the admitted jobs' paths that no wave has taken yet and
// launches it on slot W, its accumulate ordered behind prev_acc.
//
// Policy 0: jobs with the fewest remaining paths first, each taking what it
// still needs up to the capacity left.  Small jobs finish in the next wave (low
// latency); the largest share whatever remains, so the queue is always full
// (throughput).  Policy 1: an equal share per running job, then the rest in
// admission order.
static xtgpu_status launch_wave(xtgpu_service *v, WaveSlot &W, cudaEvent_t prev_acc)
{
    const int64_t cap = W.R.cap;
    W.wave.clear();
    W.ids.clear();
    int64_t left = cap;
    const int n = (int)v->active.size();
    std::vector<int> order(n);
    for (int k = 0; k < n; ++k) order[k] = k;
    std::vector<int64_t> take(n, 0);
    if (v->o.policy == 1) {
        const int64_t share = std::max<int64_t>(1, cap / n);
        for (int k = 0; k < n && left > 0; ++k) {
            SvcJob &J = v->jobs[v->active[k]];
            take[k] = std::min<int64_t>({share, J.paths - J.planned, left});
            left -= take[k];
        }
    } else {
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            const SvcJob &A = v->jobs[v->active[a]], &B = v->jobs[v->active[b]];
            return (A.paths - A.planned) < (B.paths - B.planned);
        });
    }
    for (int k : order) {
        if (left <= 0) break;
        SvcJob &J = v->jobs[v->active[k]];
        int64_t more = std::min<int64_t>(J.paths - J.planned - take[k], left);
        take[k] += more;
        left -= more;
    }
    int bounces = 0;
    for (int k = 0; k < n; ++k) {
        if (take[k] <= 0) continue;
        SvcJob &J = v->jobs[v->active[k]];
        DevJob dj{};
        dj.integrator = J.d.integrator;
        dj.width = J.d.width;
        dj.height = J.d.height;
        set_samples(dj, J.d.spp, J.d.aa, J.d.sample_distribution);
        dj.rdepth = J.d.rdepth;
        dj.ao_maxd = J.d.ao_max_distance;
        dj.seed = J.d.seed;
        dj.x0 = 0;
        dj.y0 = 0;
        dj.rw = J.d.width;
        dj.rh = J.d.height;
        dj.scene = J.d.scene;
        dj.bounces = bounces_of(J.d.integrator, J.d.rdepth);
        dj.tile = scene_tuning(v->scenes[J.d.scene]).tile;
        dj.frame = J.frame;
        dj.first = J.planned;
        dj.count = take[k];
        J.planned += take[k];
        bounces = std::max(bounces, dj.bounces);
        W.wave.push_back(dj);
        W.ids.push_back(v->active[k]);
    }
    // launch configuration: the tuning of the scene with the most paths in the
    // wave (its own if autotuned); the stack holds the deepest BVH the wave touches
    {
        std::vector<int64_t> per(v->scenes.size(), 0);
        for (const DevJob &dj : W.wave) per[dj.scene] += dj.count;
        int top = (int)(std::max_element(per.begin(), per.end()) - per.begin());
        W.R.T = scene_tuning(v->scenes[top]);
        int stack = 32;
        for (size_t k = 0; k < per.size(); ++k)
            if (per[k] > 0)
                stack = std::max(stack, stack_for_scene(v->scenes[k], v->o.node_format,
                                                        scene_tuning(v->scenes[k]).stack_entries));
        W.R.stack = stack;
        // first pass in its own format if every scene of the wave has it
        const int pf = W.R.T.primary_node_format;
        W.R.fmt0 = -1;
        if (pf >= 0 && pf != v->o.node_format) {
            bool ok = true;
            int st0 = 32;
            for (size_t k = 0; k < per.size(); ++k)
                if (per[k] > 0) {
                    ok = ok && format_built(v->scenes[k], pf);
                    st0 = std::max(st0, stack_for_scene(v->scenes[k], pf, scene_tuning(v->scenes[k]).stack_entries));
                }
            if (ok) {
                W.R.fmt0 = pf;
                W.R.stack0 = st0;
            }
        }
    }
    // frames of newly admitted jobs are allocated and zeroed on the service stream
    XTG_CUDA(cudaEventRecord(v->admitted, v->s));
    XTG_CUDA(cudaStreamWaitEvent(W.s, v->admitted, 0));
    W.R.prev_acc = prev_acc;
    XTG_TRY(W.R.run_wave(W.wave, bounces, v->o.node_format, v->o.use_graphs != 0, W.s));
    XTG_CUDA(cudaMemcpyAsync(W.jrays, W.R.q.job_rays, sizeof(unsigned long long) * W.wave.size(),
                             cudaMemcpyDeviceToHost, W.s));
    XTG_CUDA(cudaEventRecord(W.fin, W.s));
    ++v->waves;
    return XTGPU_OK;
}

// Waits for the wave on slot W, credits its paths and rays to its jobs and
// finishes the jobs it completed.  Waves retire in launch order, so a job is
// complete once the wave that took its last paths retires.
static xtgpu_status retire_wave(xtgpu_service *v, WaveSlot &W)
{
    XTG_CUDA(cudaEventSynchronize(W.fin));
    XTG_TRY(W.R.collect_times(W.s));
    double now = v->now();
    for (size_t k = 0; k < W.ids.size(); ++k) {
        SvcJob &J = v->jobs[W.ids[k]];
        J.done += W.wave[k].count;
        J.rays += W.jrays[k];
        if (J.done < J.paths) continue;
        J.render_done_s = now;
        v->active.erase(std::find(v->active.begin(), v->active.end(), W.ids[k]));
        if (v->o.host_results) {
            // frame -> pinned host memory on the service stream; the device
            // frame is freed behind the copy, so its budget is free at once
            // pinned frames come in power-of-two size classes (from 64 KB) and
            // are reused by any job whose frame fits in at most twice its
            // size: pinning memory is slow and may wait for the device, so a
            // stream of varied frame sizes should reach a steady pool, and a
            // class that runs out is pinned 64 MB (up to 16 frames) at a time
            const uint64_t cls = pinned_class(J.frame_bytes);
            auto it = v->pinned_free.lower_bound(J.frame_bytes);
            if (it != v->pinned_free.end() && it->first <= 2 * cls) {
                J.host = it->second;
                J.host_bytes = it->first;
                v->pinned_free.erase(it);
            } else {
                const uint64_t nbuf = std::max<uint64_t>(1, std::min<uint64_t>(16, (64ull << 20) / cls));
                char *chunk = nullptr;
                XTG_CUDA(cudaMallocHost((void **)&chunk, nbuf * cls));
                v->pinned_chunks.push_back(chunk);
                J.host = (float4 *)chunk;
                J.host_bytes = cls;
                for (uint64_t b = 1; b < nbuf; ++b) v->pinned_free.emplace(cls, (float4 *)(chunk + b * cls));
            }
            if (!v->events_free.empty()) {
                J.copied = v->events_free.back();
                v->events_free.pop_back();
            } else {
                XTG_CUDA(cudaEventCreateWithFlags(&J.copied, cudaEventDisableTiming));
            }
            XTG_CUDA(cudaMemcpyAsync(J.host, J.frame, J.frame_bytes, cudaMemcpyDeviceToHost, v->cs));
            XTG_CUDA(cudaFreeAsync(J.frame, v->cs));
            XTG_CUDA(cudaEventRecord(J.copied, v->cs));
            J.frame = nullptr;
            v->mem_used -= J.frame_bytes;
            v->copying.push_back(W.ids[k]);
            continue;
        }
        J.state = 2;
        J.finish_s = now;
    }
    W.wave.clear();
    W.ids.clear();
    return XTGPU_OK;
}

// Marks the jobs whose host copy has landed as done (all of them, waiting,
// when wait is set); their finish time is when the copy was seen complete.
static xtgpu_status finish_copies(xtgpu_service *v, bool wait)
{
    size_t keep = 0;
    for (size_t k = 0; k < v->copying.size(); ++k) {
        SvcJob &J = v->jobs[v->copying[k]];
        cudaError_t e = wait ? cudaEventSynchronize(J.copied) : cudaEventQuery(J.copied);
        if (e == cudaErrorNotReady) {
            v->copying[keep++] = v->copying[k];
            continue;
        }
        if (e != cudaSuccess) return cuda_fail(e, "host copy of a finished frame", __FILE__, __LINE__);
        v->events_free.push_back(J.copied);
        J.copied = nullptr;
        J.state = 2;
        J.finish_s = v->now();
    }
    v->copying.resize(keep);
    return XTGPU_OK;
}

// Waits for everything the service launched, frees its frames, runners,
// streams and events, and deletes it.
static void destroy_service(xtgpu_service *v)
{
    for (int k = 0; k < v->nslots; ++k)
        if (v->slot[k].s) cudaStreamSynchronize(v->slot[k].s);
    if (v->cs) cudaStreamSynchronize(v->cs);
    cudaStreamSynchronize(v->s);
    for (auto &kv : v->jobs) {
        if (kv.second.frame) cudaFreeAsync(kv.second.frame, v->s);
        if (kv.second.copied) cudaEventDestroy(kv.second.copied);
    }
    cudaStreamSynchronize(v->s);
    for (void *c : v->pinned_chunks) cudaFreeHost(c);
    for (cudaEvent_t e : v->events_free) cudaEventDestroy(e);
    for (int k = 0; k < v->nslots; ++k) {
        WaveSlot &W = v->slot[k];
        W.R.release();
        if (W.fin) cudaEventDestroy(W.fin);
        if (W.jrays) cudaFreeHost(W.jrays);
        if (W.s) cudaStreamDestroy(W.s);
    }
    if (v->admitted) cudaEventDestroy(v->admitted);
    if (v->cs) cudaStreamDestroy(v->cs);
    if (v->own_stream) cudaStreamDestroy(v->s);
    delete v;
}

extern "C" {

xtgpu_status xtgpu_service_create(const xtgpu_service_opts *opts, void *stream, xtgpu_service **out)
{
    if (!opts || !out || opts->max_jobs <= 0 || opts->max_jobs > 1024 || opts->wave_paths < 0 ||
        !format_valid(opts->node_format) || opts->waves_in_flight < 0 ||
        opts->waves_in_flight > XTGPU_MAX_WAVES_IN_FLIGHT) {
        set_error("xtgpu_service_create: bad options");
        return XTGPU_ERR_INVALID;
    }
    // Frames come and go with every job: keep freed pool memory cached instead
    // of returning it to the driver at each synchronisation (the default), so
    // admission does not remap memory for every job.
    {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    xtgpu_service *v = new xtgpu_service();
    v->o = *opts;
    v->s = (cudaStream_t)stream;
    v->nslots = opts->waves_in_flight > 0 ? opts->waves_in_flight : 2;
    int64_t cap = opts->wave_paths > 0 ? opts->wave_paths : (1ll << 22);
    auto fail = [&](xtgpu_status st) {
        destroy_service(v);
        return st;
    };
    if (!v->s) {
        if (cudaStreamCreateWithFlags(&v->s, cudaStreamNonBlocking) != cudaSuccess) {
            delete v;
            set_error("xtgpu_service_create: cudaStreamCreate failed");
            return XTGPU_ERR_CUDA;
        }
        v->own_stream = true;
    }
    cudaError_t e0 = cudaEventCreateWithFlags(&v->admitted, cudaEventDisableTiming);
    if (e0 == cudaSuccess) e0 = cudaStreamCreateWithFlags(&v->cs, cudaStreamNonBlocking);
    if (e0 != cudaSuccess) return fail(cuda_fail(e0, "xtgpu_service_create: event and copy stream", __FILE__, __LINE__));
    for (int k = 0; k < v->nslots; ++k) {
        WaveSlot &W = v->slot[k];
        cudaError_t e = cudaStreamCreateWithFlags(&W.s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&W.fin, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&W.jrays, sizeof(unsigned long long) * opts->max_jobs);
        if (e != cudaSuccess) return fail(cuda_fail(e, "xtgpu_service_create: wave slot", __FILE__, __LINE__));
        xtgpu_status st = W.R.init(cap, opts->max_jobs, 64, v->s);
        if (st != XTGPU_OK) return fail(st);
        W.R.enable_job_rays(true);
        W.R.time_extend = opts->time_kernels != 0;
        W.R.enable_stats(opts->count_visits != 0);
        W.R.defer_acc = v->nslots > 1;
    }
    // queue buffers are zeroed on the service stream; waves run on the slots' streams
    e0 = cudaStreamSynchronize(v->s);
    if (e0 != cudaSuccess) return fail(cuda_fail(e0, "xtgpu_service_create: synchronize", __FILE__, __LINE__));
    v->t0 = std::chrono::steady_clock::now();
    *out = v;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_add_scene(xtgpu_service *v, xtgpu_scene *sc, int32_t *id)
{
    if (!v || !sc || !id) {
        set_error("xtgpu_service_add_scene: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    if (!format_built(sc, v->o.node_format)) {
        set_error("xtgpu_service_add_scene: the service's node format is not built for this scene");
        return XTGPU_ERR_STATE;
    }
    if (v->scenes.size() >= 64) {
        set_error("xtgpu_service_add_scene: at most 64 resident scenes");
        return XTGPU_ERR_LIMIT;
    }
    v->scenes.push_back(sc);
    v->dev.push_back(sc->dev);
    for (int k = 0; k < v->nslots; ++k) XTG_TRY(v->slot[k].R.set_scenes(v->dev.data(), (int)v->dev.size(), v->s));
    XTG_CUDA(cudaStreamSynchronize(v->s));   // the slots' streams read the scene table
    *id = (int32_t)v->scenes.size() - 1;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_update_scene(xtgpu_service *v, int32_t scene)
{
    if (!v || scene < 0 || scene >= (int32_t)v->scenes.size()) {
        set_error("xtgpu_service_update_scene: NULL service or unknown scene");
        return XTGPU_ERR_INVALID;
    }
    // waves in flight read the scene table: it changes between waves only
    for (int k = 0; k < v->nslots; ++k)
        if (v->slot[k].s) XTG_CUDA(cudaStreamSynchronize(v->slot[k].s));
    XTG_CUDA(cudaStreamSynchronize(v->s));
    v->dev[(size_t)scene] = v->scenes[(size_t)scene]->dev;
    for (int k = 0; k < v->nslots; ++k) XTG_TRY(v->slot[k].R.set_scenes(v->dev.data(), (int)v->dev.size(), v->s));
    XTG_CUDA(cudaStreamSynchronize(v->s));
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_submit(xtgpu_service *v, const xtgpu_job_desc *d, double submit_s, int64_t *id)
{
    if (!v || !d || !id) {
        set_error("xtgpu_service_submit: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    if (d->scene < 0 || d->scene >= (int32_t)v->scenes.size() || d->integrator < XTGPU_STENCIL ||
        d->integrator > XTGPU_INTEGRATOR_LAST || d->width <= 0 || d->height <= 0 || d->spp <= 0 || d->rdepth < 0 ||
        (d->integrator == XTGPU_AO && !(d->ao_max_distance > 0.f))) {
        set_error("xtgpu_service_submit: bad job");
        return XTGPU_ERR_INVALID;
    }
    if (!view_valid(v->scenes[d->scene]->dev.cam, d->width, d->height, d->aa, d->sample_distribution, d->spp)) {
        set_error("xtgpu_service_submit: sample_distribution not grid or random, aa outside 0..16 (grid) or 0..256 "
                  "(random), samples per pixel above 2^31, or a cubemap height that is not six square faces");
        return XTGPU_ERR_INVALID;
    }
    int64_t paths = (int64_t)d->width * d->height * sample_positions(d->aa, d->sample_distribution) * d->spp;
    if (paths <= 0 || paths > (1ll << 40)) {
        set_error("xtgpu_service_submit: job too large");
        return XTGPU_ERR_INVALID;
    }
    SvcJob J;
    J.d = *d;
    J.paths = paths;
    J.frame_bytes = sizeof(float4) * (uint64_t)d->width * d->height;
    {
        std::lock_guard<std::mutex> lock(v->mu);
        J.submit_s = submit_s >= 0 ? submit_s : v->now();
        int64_t jid = v->next_id++;
        // keep the pending queue ordered by arrival time (stable for equal times)
        auto it = v->pending.end();
        while (it != v->pending.begin() && v->jobs[*(it - 1)].submit_s > J.submit_s) --it;
        v->jobs[jid] = J;
        v->pending.insert(it, jid);
        *id = jid;
    }
    v->arrived.notify_all();
    return XTGPU_OK;
}

}  // extern "C"

namespace {

static xtgpu_status run_loop(xtgpu_service *v, double max_seconds)
{
    std::unique_lock<std::mutex> lk(v->mu);
    const double t_end = max_seconds > 0 ? v->now() + max_seconds : 1e300;
    // slots in flight, oldest first; `last` is the most recently launched one,
    // whose accumulate the next wave's accumulate waits for
    std::deque<int> flight;
    int last = -1;
    bool out_of_time = false;
    while (true) {
        double now = v->now();
        if (!out_of_time) XTG_TRY(admit(v, now));
        // 1. launch a wave if a slot is free and an admitted job has paths no
        //    wave has taken yet
        bool plannable = false;
        if (!out_of_time && (int)flight.size() < v->nslots)
            for (int64_t id : v->active) {
                const SvcJob &J = v->jobs[id];
                if (J.planned < J.paths) {
                    plannable = true;
                    break;
                }
            }
        if (plannable) {
            int k = 0;
            while (k < v->nslots && std::find(flight.begin(), flight.end(), k) != flight.end()) ++k;
            XTG_TRY(launch_wave(v, v->slot[k], last >= 0 ? v->slot[last].R.acc_done : nullptr));
            flight.push_back(k);
            last = k;
            continue;
        }
        // 2. retire the oldest wave in flight; other threads may submit, poll
        //    and release while the loop waits for it
        if (!flight.empty()) {
            WaveSlot &W = v->slot[flight.front()];
            flight.pop_front();
            cudaEvent_t fin = W.fin;
            lk.unlock();
            cudaError_t e = cudaEventSynchronize(fin);
            lk.lock();
            if (e != cudaSuccess) return cuda_fail(e, "xtgpu_service_run: wave", __FILE__, __LINE__);
            XTG_TRY(retire_wave(v, W));
            XTG_TRY(finish_copies(v, false));
            if (v->now() >= t_end) out_of_time = true;
            continue;
        }
        if (out_of_time) return XTGPU_ERR_TIMEOUT;
        // 3. nothing in flight and nothing to launch: wait for arrivals
        if (!v->active.empty()) {
            // every admitted job is fully planned and nothing is in flight
            set_error("xtgpu_service_run: inconsistent job state");
            return XTGPU_ERR_STATE;
        }
        if (v->pending.empty()) {
            if (!v->open) return XTGPU_OK;
            // open: wait for a submission or for the service to close
            if (now >= t_end) return XTGPU_ERR_TIMEOUT;
            XTG_TRY(finish_copies(v, false));
            v->arrived.wait_for(lk, std::chrono::duration<double>(std::min(t_end - now, 0.01)));
            continue;
        }
        double next = v->jobs[v->pending.front()].submit_s;
        if (next > now) {
            if (now >= t_end) return XTGPU_ERR_TIMEOUT;
            double dt = std::min(next, t_end) - now;
            v->arrived.wait_for(lk, std::chrono::duration<double>(std::min(dt, 0.01)));
            continue;
        }
        // the head job does not fit yet and nothing runs: cannot happen
        // (admission only blocks on memory held by running jobs)
        set_error("xtgpu_service_run: admission stalled");
        return XTGPU_ERR_STATE;
    }
}

}  // namespace

extern "C" {

xtgpu_status xtgpu_service_run(xtgpu_service *v, double max_seconds)
{
    if (!v) {
        set_error("xtgpu_service_run: NULL service");
        return XTGPU_ERR_INVALID;
    }
    if (v->scenes.empty()) {
        set_error("xtgpu_service_run: no scene");
        return XTGPU_ERR_STATE;
    }
    {
        std::lock_guard<std::mutex> lock(v->mu);
        if (v->running) {
            set_error("xtgpu_service_run: already running on another thread");
            return XTGPU_ERR_STATE;
        }
        v->running = true;
    }
    xtgpu_status st = run_loop(v, max_seconds);
    std::lock_guard<std::mutex> lock(v->mu);
    // host copies of finished frames still in flight land before returning
    xtgpu_status cst = finish_copies(v, true);
    v->running = false;
    return st != XTGPU_OK ? st : cst;
}

xtgpu_status xtgpu_service_open(xtgpu_service *v, int32_t open)
{
    if (!v) {
        set_error("xtgpu_service_open: NULL service");
        return XTGPU_ERR_INVALID;
    }
    {
        std::lock_guard<std::mutex> lock(v->mu);
        v->open = open != 0;
    }
    v->arrived.notify_all();
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_poll(xtgpu_service *v, int64_t id, xtgpu_job_status *st)
{
    if (!v || !st) {
        set_error("xtgpu_service_poll: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(v->mu);
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) {
        set_error("xtgpu_service_poll: unknown job");
        return XTGPU_ERR_NOT_FOUND;
    }
    const SvcJob &J = it->second;
    st->state = J.state;
    st->rays = J.rays;
    st->submit_s = J.submit_s;
    st->start_s = J.start_s;
    st->finish_s = J.finish_s;
    st->render_done_s = J.render_done_s;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_result(xtgpu_service *v, int64_t id, float *rgba)
{
    if (!v || !rgba) {
        set_error("xtgpu_service_result: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    const float4 *frame = nullptr;
    uint64_t bytes = 0;
    {
        std::lock_guard<std::mutex> lock(v->mu);
        auto it = v->jobs.find(id);
        if (it == v->jobs.end()) {
            set_error("xtgpu_service_result: unknown job");
            return XTGPU_ERR_NOT_FOUND;
        }
        SvcJob &J = it->second;
        if (J.state == 2 && J.host) {
            memcpy(rgba, J.host, J.frame_bytes);
            return XTGPU_OK;
        }
        if (J.state != 2 || !J.frame) {
            set_error("xtgpu_service_result: job not finished or released");
            return XTGPU_ERR_STATE;
        }
        frame = J.frame;
        bytes = J.frame_bytes;
    }
    // the frame stays until this job is released (by the caller)
    XTG_CUDA(cudaMemcpyAsync(rgba, frame, bytes, cudaMemcpyDeviceToHost, v->s));
    XTG_CUDA(cudaStreamSynchronize(v->s));
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_result_host(xtgpu_service *v, int64_t id, const float **rgba)
{
    if (!v || !rgba) {
        set_error("xtgpu_service_result_host: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(v->mu);
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) {
        set_error("xtgpu_service_result_host: unknown job");
        return XTGPU_ERR_NOT_FOUND;
    }
    const SvcJob &J = it->second;
    if (J.state != 2 || !J.host) {
        set_error("xtgpu_service_result_host: no host copy (job not finished, released, or host_results off)");
        return XTGPU_ERR_STATE;
    }
    *rgba = (const float *)J.host;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_release(xtgpu_service *v, int64_t id)
{
    if (!v) {
        set_error("xtgpu_service_release: NULL service");
        return XTGPU_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(v->mu);
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) {
        set_error("xtgpu_service_release: unknown job");
        return XTGPU_ERR_NOT_FOUND;
    }
    SvcJob &J = it->second;
    if (J.state == 1) {
        set_error("xtgpu_service_release: job still running");
        return XTGPU_ERR_STATE;
    }
    if (J.frame) {
        XTG_CUDA(cudaFreeAsync(J.frame, v->s));
        J.frame = nullptr;
        v->mem_used -= J.frame_bytes;
    }
    if (J.host) {
        v->pinned_free.emplace(J.host_bytes, J.host);
        J.host = nullptr;
    }
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_get_stats(xtgpu_service *v, xtgpu_service_stats *st)
{
    if (!v || !st) {
        set_error("xtgpu_service_get_stats: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(v->mu);
    *st = xtgpu_service_stats{};
    for (int k = 0; k < v->nslots; ++k) {
        WaveRunner &R = v->slot[k].R;
        unsigned long long rays = 0, sv[2] = {0, 0};
        XTG_TRY(R.read_ctl(nullptr, &rays, v->slot[k].s));
        XTG_CUDA(cudaMemcpy(sv, R.statsbuf.p, 16, cudaMemcpyDeviceToHost));
        st->rays += rays;
        st->kernel_launches += (uint64_t)R.launches;
        st->extend_ms += R.extend_ms;
        st->extend_launches += (uint64_t)R.extend_launches;
        st->node_visits += sv[0];
        st->prim_tests += sv[1];
    }
    st->waves = v->waves;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_reset_stats(xtgpu_service *v)
{
    if (!v) {
        set_error("xtgpu_service_reset_stats: NULL service");
        return XTGPU_ERR_INVALID;
    }
    for (int k = 0; k < v->nslots; ++k) {
        WaveRunner &R = v->slot[k].R;
        XTG_CUDA(cudaStreamSynchronize(v->slot[k].s));
        XTG_CUDA(cudaMemset((char *)R.ctlbuf.p + 32, 0, 8));
        XTG_CUDA(cudaMemset(R.statsbuf.p, 0, 16));
        R.launches = 0;
        R.extend_ms = 0.0;
        R.extend_launches = 0;
    }
    v->waves = 0;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_destroy(xtgpu_service *v)
{
    if (v) destroy_service(v);
    return XTGPU_OK;
}

}  // extern "C"
