// xtgpu_render_tile_noalloc: the xtgpu_render kernels for one rectangle, with
// every scratch buffer in one file-scope static device array instead of
// memory allocated per call.
//
// For callers that cannot allocate device memory at render time: a
// render_tile running on XTracer's OpenMP tile threads, where a cudaMalloc
// would synchronise the device and stall the tiles of every other thread;
// processes that reserve their device memory at start-up under a fixed
// budget (or leave it all to another allocator) and must not allocate later;
// render loops that must not meet an allocation failure or its latency
// mid-frame.  The caller passes the scene (created beforehand) and the output
// frame; this entry point calls no cudaMalloc, cudaFree or other allocating
// routine.
//
// Limits and sharing:
//   * at most XTGPU_NOALLOC_MAX_PATHS (65536) paths per call, i.e. rectangle
//     pixels x aa^2 x spp (one 32x32 tile at 64 spp); larger requests are rejected
//     with XTGPU_ERR_LIMIT;
//   * the array (NOALLOC_BYTES, about 11.5 MB) is held by every GPU that loads
//     the library, until the process exits;
//   * all calls share it: the counters it holds are reset at the start of each
//     call, but calls that overlap on the GPU (other threads or streams) race
//     on it and corrupt each other's results;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device); make that first call before any
//     stream capture;
//   * every call copies its job from host memory and waits for its stream
//     before it returns, so the stream it is given must not be capturing
//     (XTGPU_ERR_STATE).
#include <mutex>

#include "render.h"

namespace xtg {
namespace {

constexpr int64_t NA_PATHS = XTGPU_NOALLOC_MAX_PATHS;
constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t SZ_F4 = al(sizeof(float4) * NA_PATHS);
constexpr size_t SZ_U2 = al(sizeof(uint2) * NA_PATHS);
constexpr size_t SZ_HIT = al(sizeof(xtgpu_hit) * NA_PATHS);
constexpr size_t SIDE = 4 * SZ_F4 + SZ_U2;          // org, dir, P, I, meta of one queue
constexpr size_t OFF_HIT = 2 * SIDE;
constexpr size_t OFF_CONTRIB = OFF_HIT + SZ_HIT;
constexpr size_t OFF_CTL = OFF_CONTRIB + SZ_F4;     // 64 bytes of counters (+ rays at byte 32)
constexpr size_t OFF_JOB = OFF_CTL + 256;
constexpr size_t OFF_PREFIX = OFF_JOB + al(sizeof(DevJob));
constexpr size_t OFF_SCENE = OFF_PREFIX + 256;
constexpr size_t NOALLOC_BYTES = OFF_SCENE + al(sizeof(DevScene));

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current.  In host code the symbol names a host-side stand-in, not
// device memory, so it is never passed to a kernel directly.
static std::mutex g_na_mu;
static unsigned char *g_na_addr[64] = {};
// One call at a time per device owns the scratch: tiles rendered concurrently
// from several host threads take turns (each call ends synchronised).
static std::mutex g_na_call_mu[64];

static xtgpu_status noalloc_scratch(unsigned char **out, int *device)
{
    int dev = 0;
    XTG_CUDA(cudaGetDevice(&dev));
    *device = dev;
    if (dev < 0 || dev >= 64) {
        set_error("xtgpu_render_tile_noalloc: device index out of range");
        return XTGPU_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_na_addr[dev] = (unsigned char *)p;
    }
    *out = g_na_addr[dev];
    return XTGPU_OK;
}

}  // namespace xtg

using namespace xtg;

extern "C" xtgpu_status xtgpu_render_tile_noalloc(xtgpu_scene *sc, const xtgpu_render_params *p, float *rgba,
                                                  uint64_t *rays, void *stream)
{
    if (!sc || !p || !rgba) {
        set_error("xtgpu_render_tile_noalloc: NULL argument");
        return XTGPU_ERR_INVALID;
    }
    if (p->integrator < XTGPU_STENCIL || p->integrator > XTGPU_INTEGRATOR_LAST || p->width <= 0 || p->height <= 0 ||
        p->spp <= 0 || p->rdepth < 0 || (p->integrator == XTGPU_AO && !(p->ao_max_distance > 0.f))) {
        set_error("xtgpu_render_tile_noalloc: bad parameters");
        return XTGPU_ERR_INVALID;
    }
    if (!view_valid(sc->dev.cam, p->width, p->height, p->aa, p->sample_distribution, p->spp)) {
        set_error("xtgpu_render_tile_noalloc: sample_distribution not grid or random, aa outside 0..16 (grid) or "
                  "0..256 (random), samples per pixel above 2^31, or a cubemap height that is not six square faces");
        return XTGPU_ERR_INVALID;
    }
    int x0 = p->x0, y0 = p->y0, x1 = p->x1, y1 = p->y1;
    if (x1 == 0 && y1 == 0) {
        x0 = y0 = 0;
        x1 = p->width;
        y1 = p->height;
    }
    if (x0 < 0 || y0 < 0 || x1 > p->width || y1 > p->height || x0 >= x1 || y0 >= y1) {
        set_error("xtgpu_render_tile_noalloc: bad rectangle");
        return XTGPU_ERR_INVALID;
    }
    const int64_t npix = (int64_t)(x1 - x0) * (y1 - y0);
    const int64_t paths = npix * sample_positions(p->aa, p->sample_distribution) * p->spp;
    if (paths > NA_PATHS) {
        set_error("xtgpu_render_tile_noalloc: rectangle pixels x positions x spp exceeds the 65536-path scratch array; "
                  "split the frame into smaller tiles");
        return XTGPU_ERR_LIMIT;
    }
    if (!format_valid(p->node_format) || !format_built(sc, p->node_format)) {
        set_error("xtgpu_render_tile_noalloc: node format not built for this scene");
        return XTGPU_ERR_STATE;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    XTG_CUDA(cudaStreamIsCapturing((cudaStream_t)stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("xtgpu_render_tile_noalloc: the stream is capturing; each call copies its job from host memory "
                  "and waits for the stream");
        return XTGPU_ERR_STATE;
    }
    unsigned char *base = nullptr;
    int dev = 0;
    XTG_TRY(noalloc_scratch(&base, &dev));
    std::lock_guard<std::mutex> call_lock(g_na_call_mu[dev]);
    cudaStream_t s = (cudaStream_t)stream;

    WaveQueues q{};
    for (int k = 0; k < 2; ++k) {
        unsigned char *side = base + k * SIDE;
        q.org[k] = (float4 *)(side);
        q.dir[k] = (float4 *)(side + SZ_F4);
        q.P[k] = (float4 *)(side + 2 * SZ_F4);
        q.I[k] = (float4 *)(side + 3 * SZ_F4);
        q.meta[k] = (uint2 *)(side + 4 * SZ_F4);
    }
    q.hit = (xtgpu_hit *)(base + OFF_HIT);
    q.contrib = (float4 *)(base + OFF_CONTRIB);
    q.ctl = (int32_t *)(base + OFF_CTL);
    q.rays = (unsigned long long *)(base + OFF_CTL + 32);
    q.job_rays = nullptr;
    q.stats = nullptr;
    q.capacity = NA_PATHS;
    DevJob *jobs_dev = (DevJob *)(base + OFF_JOB);
    int64_t *prefix_dev = (int64_t *)(base + OFF_PREFIX);
    DevScene *scene_dev = (DevScene *)(base + OFF_SCENE);

    DevJob J{};
    J.integrator = p->integrator;
    J.width = p->width;
    J.height = p->height;
    set_samples(J, p->spp, p->aa, p->sample_distribution);
    J.rdepth = p->rdepth;
    J.ao_maxd = p->ao_max_distance;
    J.seed = p->seed;
    J.x0 = x0;
    J.y0 = y0;
    J.rw = x1 - x0;
    J.rh = y1 - y0;
    J.scene = 0;
    J.bounces = bounces_of(p->integrator, p->rdepth);
    const xtgpu_tuning &T = scene_tuning(sc);
    J.tile = T.tile;
    J.frame = (float4 *)rgba;
    J.first = 0;
    J.count = paths;
    J.offset = 0;
    const int64_t prefix[2] = {0, npix < paths ? npix : paths};
    // every counter starts at zero on each call; the array keeps the last
    // call's contents otherwise
    int32_t ctl[16] = {0};
    ctl[0] = (int32_t)paths;
    ctl[4] = 1;
    ctl[5] = (int32_t)paths;
    XTG_CUDA(cudaMemcpyAsync(jobs_dev, &J, sizeof(DevJob), cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(prefix_dev, prefix, sizeof(prefix), cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(scene_dev, &sc->dev, sizeof(DevScene), cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(q.ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemsetAsync(rgba, 0, sizeof(float4) * npix, s));
    int sms = 148;
    XTG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // the camera rays take the tuned node format when it is built, as in xtgpu_render
    int fmt0 = -1, stack0 = 0;
    if (T.primary_node_format >= 0 && T.primary_node_format != p->node_format &&
        format_built(sc, T.primary_node_format)) {
        fmt0 = T.primary_node_format;
        stack0 = stack_for_scene(sc, fmt0, T.stack_entries);
    }
    enqueue_wave_raw(T, q, jobs_dev, scene_dev, sc->dev, prefix_dev, J.bounces, p->node_format, sms,
                     stack_for_scene(sc, p->node_format, T.stack_entries), fmt0, stack0, s);
    XTG_CUDA(cudaGetLastError());
    int32_t back[16];
    XTG_CUDA(cudaMemcpyAsync(back, q.ctl, sizeof(back), cudaMemcpyDeviceToHost, s));
    XTG_CUDA(cudaStreamSynchronize(s));
    if (rays) *rays = *(const unsigned long long *)((const char *)back + 32);
    if (back[3]) {
        set_error("xtgpu_render_tile_noalloc: traversal stack overflow");
        return XTGPU_ERR_LIMIT;
    }
    return XTGPU_OK;
}
