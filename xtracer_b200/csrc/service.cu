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
// Because paths are keyed by (seed, pixel, sample) and folded per pixel in
// sample order, a job's frame is bit-identical whatever it is merged with.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <vector>

#include "render.h"

namespace xtg {

struct SvcJob {
    xtgpu_job_desc d{};
    int state = 0;   // 0 queued, 1 running, 2 done, 3 failed
    double submit_s = 0, start_s = 0, finish_s = 0;
    int64_t paths = 0, done = 0;
    uint64_t rays = 0;
    uint64_t frame_bytes = 0;
    float4 *frame = nullptr;
    std::vector<float4> host;   // host copy (host_results)
};

}  // namespace xtg

struct xtgpu_service {
    xtgpu_service_opts o{};
    cudaStream_t s = nullptr;
    bool own_stream = false;   // created here: the legacy default stream cannot be captured
    xtg::WaveRunner R;
    std::vector<xtgpu_scene *> scenes;
    std::vector<xtg::DevScene> dev;
    std::map<int64_t, xtg::SvcJob> jobs;
    std::deque<int64_t> pending;     // submitted, not admitted (FIFO)
    std::vector<int64_t> active;     // admitted, not finished (admission order)
    int64_t next_id = 0;
    uint64_t mem_used = 0;
    std::chrono::steady_clock::time_point t0;
    std::vector<unsigned long long> wave_rays;
    uint64_t waves = 0;

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

extern "C" {

xtgpu_status xtgpu_service_create(const xtgpu_service_opts *opts, void *stream, xtgpu_service **out)
{
    if (!opts || !out || opts->max_jobs <= 0 || opts->max_jobs > 1024 || opts->wave_paths < 0 ||
        (opts->node_format != XTGPU_NODES_FP32 && opts->node_format != XTGPU_NODES_Q8)) {
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
    if (!v->s) {
        if (cudaStreamCreateWithFlags(&v->s, cudaStreamNonBlocking) != cudaSuccess) {
            delete v;
            set_error("xtgpu_service_create: cudaStreamCreate failed");
            return XTGPU_ERR_CUDA;
        }
        v->own_stream = true;
    }
    int64_t cap = opts->wave_paths > 0 ? opts->wave_paths : (1ll << 22);
    xtgpu_status st = v->R.init(cap, opts->max_jobs, 64, v->s);
    if (st != XTGPU_OK) {
        v->R.release();
        if (v->own_stream) cudaStreamDestroy(v->s);
        delete v;
        return st;
    }
    v->R.enable_job_rays(true);
    v->R.time_extend = opts->time_kernels != 0;
    v->R.enable_stats(opts->count_visits != 0);
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
    if ((v->o.node_format == XTGPU_NODES_FP32 && !sc->built32) || (v->o.node_format == XTGPU_NODES_Q8 && !sc->built8)) {
        set_error("xtgpu_service_add_scene: the service's node format is not built for this scene");
        return XTGPU_ERR_STATE;
    }
    if (v->scenes.size() >= 64) {
        set_error("xtgpu_service_add_scene: at most 64 resident scenes");
        return XTGPU_ERR_LIMIT;
    }
    v->scenes.push_back(sc);
    v->dev.push_back(sc->dev);
    XTG_TRY(v->R.set_scenes(v->dev.data(), (int)v->dev.size(), v->s));
    *id = (int32_t)v->scenes.size() - 1;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_submit(xtgpu_service *v, const xtgpu_job_desc *d, double submit_s, int64_t *id)
{
    if (!v || !d || !id) {
        set_error("xtgpu_service_submit: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    if (d->scene < 0 || d->scene >= (int32_t)v->scenes.size() || d->integrator < XTGPU_STENCIL ||
        d->integrator > XTGPU_PATHTRACER || d->width <= 0 || d->height <= 0 || d->spp <= 0 || d->rdepth < 0 ||
        (d->integrator == XTGPU_AO && !(d->ao_max_distance > 0.f))) {
        set_error("xtgpu_service_submit: bad job");
        return XTGPU_ERR_INVALID;
    }
    int64_t paths = (int64_t)d->width * d->height * d->spp;
    if (paths <= 0 || paths > (1ll << 40)) {
        set_error("xtgpu_service_submit: job too large");
        return XTGPU_ERR_INVALID;
    }
    SvcJob J;
    J.d = *d;
    J.submit_s = submit_s >= 0 ? submit_s : v->now();
    J.paths = paths;
    J.frame_bytes = sizeof(float4) * (uint64_t)d->width * d->height;
    int64_t jid = v->next_id++;
    // keep the pending queue ordered by arrival time (stable for equal times)
    auto it = v->pending.end();
    while (it != v->pending.begin() && v->jobs[*(it - 1)].submit_s > J.submit_s) --it;
    v->jobs[jid] = J;
    v->pending.insert(it, jid);
    *id = jid;
    return XTGPU_OK;
}

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
    const double t_end = max_seconds > 0 ? v->now() + max_seconds : 1e300;
    const int64_t cap = v->R.cap;
    std::vector<DevJob> wave;
    std::vector<int64_t> ids;
    while (true) {
        double now = v->now();
        XTG_TRY(admit(v, now));
        if (v->active.empty()) {
            if (v->pending.empty()) return XTGPU_OK;
            double next = v->jobs[v->pending.front()].submit_s;
            if (next > now) {
                if (now >= t_end) return XTGPU_ERR_TIMEOUT;
                double dt = std::min(next, t_end) - now;
                std::this_thread::sleep_for(std::chrono::duration<double>(std::min(dt, 0.01)));
                continue;
            }
            // the head job does not fit yet and nothing runs: cannot happen
            // (admission only blocks on memory held by running jobs)
            set_error("xtgpu_service_run: admission stalled");
            return XTGPU_ERR_STATE;
        }
        // plan the wave: jobs with the fewest remaining paths first, each taking
        // what it still needs up to the capacity left.  Small jobs finish in the
        // next wave (low latency); the largest share whatever remains, so the
        // queue is always full (throughput).
        wave.clear();
        ids.clear();
        int64_t left = cap;
        int n = (int)v->active.size();
        std::vector<int> order(n);
        for (int k = 0; k < n; ++k) order[k] = k;
        std::vector<int64_t> take(n, 0);
        if (v->o.policy == 1) {
            // equal share per running job, then the rest in admission order
            const int64_t share = std::max<int64_t>(1, cap / n);
            for (int k = 0; k < n && left > 0; ++k) {
                SvcJob &J = v->jobs[v->active[k]];
                take[k] = std::min<int64_t>({share, J.paths - J.done, left});
                left -= take[k];
            }
        } else {
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
                const SvcJob &A = v->jobs[v->active[a]], &B = v->jobs[v->active[b]];
                return (A.paths - A.done) < (B.paths - B.done);
            });
        }
        for (int k : order) {
            if (left <= 0) break;
            SvcJob &J = v->jobs[v->active[k]];
            int64_t more = std::min<int64_t>(J.paths - J.done - take[k], left);
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
            dj.spp = J.d.spp;
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
            dj.first = J.done;
            dj.count = take[k];
            bounces = std::max(bounces, dj.bounces);
            wave.push_back(dj);
            ids.push_back(v->active[k]);
        }
        // launch configuration: the tuning of the scene with the most paths in
        // the wave (its own if autotuned); the stack holds the deepest BVH the
        // wave touches
        {
            std::vector<int64_t> per(v->scenes.size(), 0);
            for (const DevJob &dj : wave) per[dj.scene] += dj.count;
            int top = (int)(std::max_element(per.begin(), per.end()) - per.begin());
            v->R.T = scene_tuning(v->scenes[top]);
            int stack = 32;
            for (size_t k = 0; k < per.size(); ++k)
                if (per[k] > 0)
                    stack = std::max(stack, stack_for_depth(v->scenes[k]->depth, scene_tuning(v->scenes[k]).stack_entries));
            v->R.stack = stack;
        }
        XTG_TRY(v->R.run_wave(wave, bounces, v->o.node_format, v->o.use_graphs != 0, v->s));
        v->wave_rays.resize(wave.size());
        XTG_CUDA(cudaMemcpyAsync(v->wave_rays.data(), v->R.q.job_rays, sizeof(unsigned long long) * wave.size(),
                                 cudaMemcpyDeviceToHost, v->s));
        XTG_CUDA(cudaStreamSynchronize(v->s));
        XTG_TRY(v->R.collect_times(v->s));
        ++v->waves;
        now = v->now();
        for (size_t k = 0; k < ids.size(); ++k) {
            SvcJob &J = v->jobs[ids[k]];
            J.done += wave[k].count;
            J.rays += v->wave_rays[k];
            if (J.done >= J.paths) {
                if (v->o.host_results) {
                    J.host.resize((size_t)J.d.width * J.d.height);
                    XTG_CUDA(cudaMemcpyAsync(J.host.data(), J.frame, J.frame_bytes, cudaMemcpyDeviceToHost, v->s));
                    XTG_CUDA(cudaFreeAsync(J.frame, v->s));
                    XTG_CUDA(cudaStreamSynchronize(v->s));
                    J.frame = nullptr;
                    v->mem_used -= J.frame_bytes;
                    now = v->now();
                }
                J.state = 2;
                J.finish_s = now;
                v->active.erase(std::find(v->active.begin(), v->active.end(), ids[k]));
            }
        }
        if (now >= t_end) return XTGPU_ERR_TIMEOUT;
    }
}

xtgpu_status xtgpu_service_poll(xtgpu_service *v, int64_t id, xtgpu_job_status *st)
{
    if (!v || !st) {
        set_error("xtgpu_service_poll: NULL argument");
        return XTGPU_ERR_INVALID;
    }
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
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_result(xtgpu_service *v, int64_t id, float *rgba)
{
    if (!v || !rgba) {
        set_error("xtgpu_service_result: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) {
        set_error("xtgpu_service_result: unknown job");
        return XTGPU_ERR_NOT_FOUND;
    }
    SvcJob &J = it->second;
    if (J.state == 2 && !J.host.empty()) {
        memcpy(rgba, J.host.data(), J.frame_bytes);
        return XTGPU_OK;
    }
    if (J.state != 2 || !J.frame) {
        set_error("xtgpu_service_result: job not finished or released");
        return XTGPU_ERR_STATE;
    }
    XTG_CUDA(cudaMemcpyAsync(rgba, J.frame, J.frame_bytes, cudaMemcpyDeviceToHost, v->s));
    XTG_CUDA(cudaStreamSynchronize(v->s));
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_release(xtgpu_service *v, int64_t id)
{
    if (!v) {
        set_error("xtgpu_service_release: NULL service");
        return XTGPU_ERR_INVALID;
    }
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
    std::vector<float4>().swap(J.host);
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_get_stats(xtgpu_service *v, xtgpu_service_stats *st)
{
    if (!v || !st) {
        set_error("xtgpu_service_get_stats: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    unsigned long long rays = 0, sv[2] = {0, 0};
    XTG_TRY(v->R.read_ctl(nullptr, &rays, v->s));
    XTG_CUDA(cudaMemcpy(sv, v->R.statsbuf.p, 16, cudaMemcpyDeviceToHost));
    st->rays = rays;
    st->waves = v->waves;
    st->kernel_launches = (uint64_t)v->R.launches;
    st->extend_ms = v->R.extend_ms;
    st->extend_launches = (uint64_t)v->R.extend_launches;
    st->node_visits = sv[0];
    st->prim_tests = sv[1];
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_reset_stats(xtgpu_service *v)
{
    if (!v) {
        set_error("xtgpu_service_reset_stats: NULL service");
        return XTGPU_ERR_INVALID;
    }
    XTG_CUDA(cudaStreamSynchronize(v->s));
    XTG_CUDA(cudaMemset((char *)v->R.ctlbuf.p + 32, 0, 8));
    XTG_CUDA(cudaMemset(v->R.statsbuf.p, 0, 16));
    v->waves = 0;
    v->R.launches = 0;
    v->R.extend_ms = 0.0;
    v->R.extend_launches = 0;
    return XTGPU_OK;
}

xtgpu_status xtgpu_service_destroy(xtgpu_service *v)
{
    if (!v) return XTGPU_OK;
    cudaStreamSynchronize(v->s);
    for (auto &kv : v->jobs)
        if (kv.second.frame) cudaFreeAsync(kv.second.frame, v->s);
    cudaStreamSynchronize(v->s);
    v->R.release();
    if (v->own_stream) cudaStreamDestroy(v->s);
    delete v;
    return XTGPU_OK;
}

}  // extern "C"
