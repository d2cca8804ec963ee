// Autotuner: per scene, the knobs that the best launch shape and data layout
// depend on — primitives per BVH leaf, extend kernel (warp-batched or pooled
// lanes, and how often the pool votes), traversal stack size, camera tile,
// register cap of the extend kernel and wave size — picked by timing a probe
// pathtracer job for each candidate of one knob at a time (coordinate descent
// from the process-wide tuning).  No counterpart in the reference, which has
// fixed octree limits (mesh.h:11-12) and a fixed 32-pixel tile (context.cc:5).
#include <chrono>
#include <vector>

#include "render.h"

using namespace xtg;

namespace {

// A candidate replaces the current setting only when its probe is at least 2 %
// faster: the probe's run-to-run spread is a few per cent, and a pick made on
// noise (a smaller wave, another builder) can cost more on a served stream
// than it gained on the probe.
constexpr float kGain = 0.98f;

struct Probe {
    xtgpu_scene *sc;
    int fmt;
    float *frame;
    cudaStream_t s;
    cudaEvent_t e0, e1;
};

// best of two timed runs after one warm-up, in ms of device time
xtgpu_status probe_ms(Probe &P, const xtgpu_tuning &T, float *ms)
{
    xtgpu_render_params p{};
    p.integrator = XTGPU_PATHTRACER;
    p.width = 512;
    p.height = 512;
    p.spp = 4;
    p.rdepth = 4;
    p.ao_max_distance = 100.f;
    p.seed = 97;
    p.node_format = P.fmt;
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        XTG_CUDA(cudaEventRecord(P.e0, P.s));
        XTG_TRY(render_impl(P.sc, &p, P.frame, nullptr, P.s, T));
        XTG_CUDA(cudaEventRecord(P.e1, P.s));
        XTG_CUDA(cudaEventSynchronize(P.e1));
        float t = 0.f;
        XTG_CUDA(cudaEventElapsedTime(&t, P.e0, P.e1));
        if (r > 0 && t < best) best = t;
    }
    *ms = best;
    return XTGPU_OK;
}

xtgpu_status rebuild(xtgpu_scene *sc, int fmt, int leaf, int layout, int builder, cudaStream_t s)
{
    sc->built32 = sc->built8 = sc->builtW = false;   // force a new topology
    XTG_TRY(build_bvh(sc, XTGPU_NODES_FP32, leaf, layout, s, builder));
    if (fmt != XTGPU_NODES_FP32) XTG_TRY(build_bvh(sc, fmt, leaf, layout, s, builder));
    return XTGPU_OK;
}

}  // namespace

extern "C" xtgpu_status xtgpu_autotune(xtgpu_scene *sc, int32_t fmt, double budget_ms, xtgpu_tuning *best,
                                       void *stream)
{
    if (!sc || !format_valid(fmt) || !(budget_ms > 0)) {
        set_error("xtgpu_autotune: bad argument");
        return XTGPU_ERR_INVALID;
    }
    if (!sc->built32) {
        set_error("xtgpu_autotune: build the scene's BVH first");
        return XTGPU_ERR_STATE;
    }
    const auto t_start = std::chrono::steady_clock::now();
    auto elapsed_ms = [&] {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    };
    cudaStream_t s = (cudaStream_t)stream;
    Probe P{sc, fmt, nullptr, s, nullptr, nullptr};
    XTG_CUDA(cudaMallocAsync((void **)&P.frame, sizeof(float4) * 512 * 512, s));
    XTG_CUDA(cudaEventCreate(&P.e0));
    XTG_CUDA(cudaEventCreate(&P.e1));
    const bool had8 = sc->built8;
    xtgpu_tuning T = scene_tuning(sc);
    xtgpu_status st = XTGPU_OK;
    float cur = 0.f;
    if (fmt != XTGPU_NODES_FP32 && !format_built(sc, fmt))
        st = build_bvh(sc, fmt, sc->leaf_size, sc->layout, s, sc->builder);
    if (st == XTGPU_OK) {
        T.leaf_size = sc->leaf_size;
        T.bvh_builder = sc->builder;
        st = probe_ms(P, T, &cur);
    }
    // 0. the hierarchy builder (rebuilds the BVH)
    if (st == XTGPU_OK && elapsed_ms() <= budget_ms) {
        const int other = 1 - T.bvh_builder;
        // a tree the other builder cannot make (too deep for the stack) keeps the first
        if (rebuild(sc, fmt, T.leaf_size, T.node_layout, other, s) != XTGPU_OK) {
            st = rebuild(sc, fmt, T.leaf_size, T.node_layout, T.bvh_builder, s);
        } else {
            xtgpu_tuning C = T;
            C.bvh_builder = other;
            float t = 0.f;
            if ((st = probe_ms(P, C, &t)) == XTGPU_OK) {
                if (t < cur * kGain) {
                    cur = t;
                    T = C;
                } else {
                    st = rebuild(sc, fmt, T.leaf_size, T.node_layout, T.bvh_builder, s);
                }
            }
        }
    }
    // 1. primitives per leaf (rebuilds the BVH)
    if (st == XTGPU_OK) {
        int best_leaf = T.leaf_size;
        for (int leaf : {1, 2, fmt == XTGPU_NODES_W8 ? 3 : 4}) {
            if (leaf == T.leaf_size || elapsed_ms() > budget_ms) continue;
            if ((st = rebuild(sc, fmt, leaf, T.node_layout, T.bvh_builder, s)) != XTGPU_OK) break;
            xtgpu_tuning C = T;
            C.leaf_size = leaf;
            float t = 0.f;
            if ((st = probe_ms(P, C, &t)) != XTGPU_OK) break;
            if (t < cur * kGain) {
                cur = t;
                best_leaf = leaf;
            }
        }
        if (st == XTGPU_OK && sc->leaf_size != best_leaf)
            st = rebuild(sc, fmt, best_leaf, T.node_layout, T.bvh_builder, s);
        T.leaf_size = best_leaf;
    }
    // 2. launch knobs, one at a time
    auto knob = [&](int32_t xtgpu_tuning::*field, std::vector<int32_t> values) {
        if (st != XTGPU_OK) return;
        int32_t keep = T.*field;
        for (int32_t v : values) {
            if (v == keep || elapsed_ms() > budget_ms) continue;
            xtgpu_tuning C = T;
            C.*field = v;
            float t = 0.f;
            if ((st = probe_ms(P, C, &t)) != XTGPU_OK) return;
            if (t < cur * kGain) {
                cur = t;
                T = C;
            }
        }
    };
    knob(&xtgpu_tuning::extend_variant, {0, 2});
    if (fmt != XTGPU_NODES_FP32 && sc->built32) knob(&xtgpu_tuning::primary_node_format, {-1, XTGPU_NODES_FP32});
    knob(&xtgpu_tuning::primary_variant, {-1, 0, 2});
    if (T.extend_variant == 2) knob(&xtgpu_tuning::steps_per_vote, {4, 8, 16});
    if ((fmt == XTGPU_NODES_W8 ? sc->depthW : sc->depth) <= 30) knob(&xtgpu_tuning::stack_entries, {32, 64});
    knob(&xtgpu_tuning::extend_min_blocks, {0, 8, 10});
    knob(&xtgpu_tuning::tile, {0, 4, 8, 16});
    if (st == XTGPU_OK) {
        // wave size: 1 Mi or 4 Mi paths.  The probe itself is one 1 Mi-path
        // job, so it cannot tell these apart by much; smaller waves lose on
        // many-job streams (grid tails, underfilled launches) and are not tried.
        int64_t keep = T.wave_paths;
        for (int64_t w : {(int64_t)1 << 20, (int64_t)1 << 22}) {
            if (w == keep || elapsed_ms() > budget_ms) continue;
            xtgpu_tuning C = T;
            C.wave_paths = w;
            float t = 0.f;
            if ((st = probe_ms(P, C, &t)) != XTGPU_OK) break;
            if (t < cur * kGain) {
                cur = t;
                T = C;
            }
        }
    }
    cudaEventDestroy(P.e0);
    cudaEventDestroy(P.e1);
    cudaFreeAsync(P.frame, s);
    if (st != XTGPU_OK) return st;
    if (!had8 && fmt != XTGPU_NODES_Q8) sc->built8 = false;
    sc->tune = T;
    sc->tuned = true;
    if (best) *best = T;
    return XTGPU_OK;
}
