// Wavefront integrators: the per-sample logic of the reference's stencil,
// depth, ao and pathtracer render_tile methods, split into queue stages.
//
//   camera     one ray per (pixel, sample) of every job in the wave
//   extend     closest hit of every queued ray (traverse.cuh)
//   shade      integrator step: contribution of finished paths, next rays of the
//              others appended to the next queue (warp-aggregated atomics)
//   accumulate per pixel, the samples of the wave folded in sample order into
//              the job's frame exactly as the reference folds them (float
//              colour channels clamped at 0, alpha clamped to [0, 1])
//
// A path's result depends only on (job seed, pixel, sample): the random stream is
// keyed by them, never by a queue slot, and the fold runs in sample order.  So a
// job renders to the same bits alone, split over any number of waves, or merged
// with other jobs.
#pragma once

#include "traverse.cuh"

namespace xtg {

// One job's share of a wave.
struct DevJob {
    int32_t integrator, width, height;
    int32_t spp;                     // samples per pixel: positions x spp1
    int32_t rdepth;
    float ao_maxd;
    uint64_t seed;
    int32_t x0, y0, rw, rh;          // rectangle rendered
    int32_t scene;                   // index in the scene table
    int32_t bounces;                 // extend passes this job needs
    int32_t tile;                    // camera order: square pixel tiles of this edge (0 = rows)
    float4 *frame;                   // rw*rh RGBA accumulation buffer
    int64_t first;                   // first path id of the job in this wave
    int64_t count;                   // paths of the job in this wave
    int64_t offset;                  // wave-local index of the job's first path
    int32_t aa;                      // anti-aliasing level (grid: 1 = pixel centre)
    int32_t spp1;                    // samples per position
    double wt;                       // weight of one sample: 1/positions as a float, times 1/spp1
    float *raygraph;                 // depth integrator: 10 floats per sample (origin, hit
                                     // point, colour after the sample), rectangle pixels
                                     // row-major, each pixel's samples in order; or null
    int32_t dist;                    // XTGPU_SAMPLES_GRID or XTGPU_SAMPLES_RANDOM
};

// Key of the random distribution's offsets of one position of one pixel: a
// stream apart from the paths' (seed ^ this salt).
constexpr uint64_t JITTER_SALT = 0xA0761D6478BD642Full;

// Positions per pixel (aa.cc:7-48): the grid's aa^2, the random
// distribution's aa; level 0 renders as level 1.
inline int sample_positions(int aa, int dist)
{
    const int L = aa > 1 ? aa : 1;
    return dist == XTGPU_SAMPLES_RANDOM ? L : L * L;
}

// Fills the sample fields of a job from params_t's samples, aa and
// sample_distribution (aa.cc:7-77): P positions of weight 1.f/P each taken
// spp times at 1/spp.
inline void set_samples(DevJob &j, int spp, int aa, int dist)
{
    const int L = aa > 1 ? aa : 1, P = sample_positions(aa, dist);
    j.aa = L;
    j.dist = dist;
    j.spp1 = spp;
    j.spp = P * spp;
    j.wt = (P == 1 ? 1.0 : (double)(1.f / (float)P)) * (1.0 / (double)spp);
}

struct WaveQueues {
    float4 *org[2], *dir[2];         // (org, tmin), (dir, tmax)
    uint2 *meta[2];                  // (wave-local path index, job slot)
    float4 *P[2];                    // (prefix throughput rgb, rng counter)
    float4 *I[2];                    // (incoming intensity rgb, depth left)
    xtgpu_hit *hit;
    float4 *contrib;                 // per wave-local path: result of the sample
    int32_t *ctl;                    // [0],[1] queue counts, [2] fetch counter, [3] overflow flag,
                                     // [4] jobs in the wave, [5] paths in the wave
    unsigned long long *rays;        // rays traced (extend inputs)
    unsigned long long *job_rays;    // per job of the wave, or nullptr
    unsigned long long *stats;       // [0] nodes visited, [1] primitives tested, or nullptr
    int64_t capacity;
};

}  // namespace xtg
