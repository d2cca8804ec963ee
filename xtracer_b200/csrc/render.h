// Host side of the wavefront: queue buffers, job table, CUDA-graph cache.
#pragma once

#include <array>
#include <map>
#include <vector>

#include "wavefront.cuh"

namespace xtg {

struct WaveRunner {
    WaveQueues q{};
    HostBuf bufs[10], hitbuf, contribbuf, ctlbuf, jobbuf, prefixbuf, scenebuf, jobraysbuf;
    bool job_rays_enabled = false;
    int32_t overflow_seen = 0;
    // live timing of the extend kernel (CUDA events around each launch, also
    // inside captured graphs) and launch counting
    static constexpr int MAX_TIMED = 16;
    bool time_extend = false;
    cudaEvent_t ev[2 * MAX_TIMED] = {};
    double extend_ms = 0.0;
    int64_t extend_launches = 0;
    int64_t launches = 0;
    int last_bounces = 0;
    HostBuf statsbuf;
    // overlapped waves: accumulate launched after the wave's graph, ordered
    // behind prev_acc (the previous wave's accumulate), signalling acc_done
    bool defer_acc = false;
    cudaEvent_t acc_done = nullptr;
    cudaEvent_t prev_acc = nullptr;
    xtgpu_status collect_times(cudaStream_t s);
    void enable_stats(bool on) { q.stats = on ? (unsigned long long *)statsbuf.p : nullptr; }
    // Pinned staging of a wave's job table, pixel prefix and counters.  The
    // copies run when the stream reaches them, after the host may already have
    // planned further waves, so two slots alternate and a slot is rewritten
    // only once its previous copies have run.
    struct Staging {
        DevJob *jobs = nullptr;
        int64_t *prefix = nullptr;
        int32_t *ctl = nullptr;            // 24 bytes used
        cudaEvent_t copied = nullptr;      // recorded after the slot's copies
        bool pending = false;
    };
    Staging stage[2];
    int stage_next = 0;
    int32_t *host_ctl = nullptr;      // pinned, 64 bytes: read_ctl
    int64_t cap = 0;
    int max_jobs = 0, max_scenes = 0, nscenes = 0;
    int sms = 148;
    DevScene single{};                 // the scene of a wave whose jobs share one
    std::vector<DevScene> host_scenes; // host copy of the scene table
    xtgpu_tuning T{};   // launch configuration of the next waves
    int stack = 64;     // traversal stack entries (32 or 64)
    int fmt0 = -1;      // node format of the first extend pass (-1 = the wave's)
    int stack0 = 64;    // its stack entries
    using GraphKey = std::array<int32_t, 17>;
    std::map<GraphKey, cudaGraphExec_t> graphs;

    xtgpu_status init(int64_t capacity, int max_jobs, int max_scenes, cudaStream_t s);
    void release();
    xtgpu_status set_scenes(const DevScene *scenes, int n, cudaStream_t s);
    // jobs[j].first/count select the job's paths in this wave; offset is filled in.
    xtgpu_status run_wave(const std::vector<DevJob> &jobs, int bounces, int fmt, bool use_graph, cudaStream_t s);
    xtgpu_status read_ctl(int32_t *overflow, unsigned long long *rays, cudaStream_t s);
    // per-job ray counts of the last wave (requires enable_job_rays)
    void enable_job_rays(bool on) { job_rays_enabled = on; q.job_rays = on ? (unsigned long long *)jobraysbuf.p : nullptr; }
    void enqueue(int njobs, int64_t total, int bounces, int fmt, bool multi, cudaStream_t s, bool capturing);
};

int bounces_of(int integrator, int rdepth);
xtgpu_tuning &tuning();
void launch_extend_kernel(const xtgpu_tuning &T, int fmt, bool multi, const DevScene &single,
                          const DevScene *scenes, const DevJob *jobs, const WaveQueues &q, int side, int sms,
                          int stack, cudaStream_t s);
// smallest stack variant (32 or 64 entries) that holds a tree of this depth
int stack_for_depth(int depth, int requested);
// One single-scene wave over caller-provided device buffers: no allocation and
// no host synchronisation.  jobs/scenes/prefix and q.ctl must already hold the
// wave (ctl[0] = ctl[5] = paths, ctl[4] = jobs, other counters zero).
void enqueue_wave_raw(const xtgpu_tuning &T, const WaveQueues &q, const DevJob *jobs, const DevScene *scenes,
                      const DevScene &single, const int64_t *prefix, int bounces, int fmt, int sms, int stack,
                      int fmt0, int stack0, cudaStream_t s);
// Closest hit of the q.ctl[side] rays of queue `side` (no job table needed).
void launch_extend(const xtgpu_tuning &T, int fmt, const DevScene &S, const WaveQueues &q, int side, int sms,
                   int stack, cudaStream_t s);

}  // namespace xtg
