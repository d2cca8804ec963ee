// 8-wide BVH with 8-bit quantised child bounds, collapsed from the binary LBVH
// on the device.  The node layout and the traversal order follow Ylitie,
// Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs" (HPG 2017); the collapse is a greedy one.
//
// Build, one kernel launch per level of the wide tree (top down):
//   * a wide node starts from one binary internal node and repeatedly opens the
//     internal child with the largest surface area until it has 8 children or
//     only leaves are left;
//   * the children take slots by direction: the child whose centroid lies
//     furthest towards octant s (relative to the node's centre) gets slot s, so
//     a ray visits slots in the order slot ^ m (m = the ray's sign bits) and
//     meets nearer children first;
//   * internal children get consecutive node indices in slot order (base + the
//     number of internal children in lower slots); the primitives of the leaf
//     children are copied next to each other (base + a 5-bit offset per child),
//     so one node names all of them.
//
// Node, 80 bytes (5 x uint4):
//   w[0..2]  origin x, y, z (float bits; the low byte holds the biased
//            power-of-two exponent of that axis' quantum)
//   w[3]     imask: bit s set if slot s is an internal child
//   w[4]     index of the first internal child
//   w[5]     index of the first leaf primitive
//   w[6..7]  meta[8]: leaf slot = (count << 5) | offset, 0 otherwise
//   w[8..19] qlo.x[8] qlo.y[8] qlo.z[8] qhi.x[8] qhi.y[8] qhi.z[8]; an unused
//            slot has qlo = 255 > qhi = 0 and is never hit
#include <algorithm>
#include <vector>

#include "xtgpu_internal.cuh"
#include "wide.cuh"

namespace xtg {

namespace {

struct WideItem {
    int32_t bref;   // binary node (>= 0) or leaf ref (< 0) the wide node starts from
    int32_t widx;   // index of the wide node
};

__device__ __forceinline__ uint32_t origin_bits_w(float v)
{
    uint32_t b = __float_as_uint(v);
    if (v == 0.f) return 0u;
    if (b & 0x80000000u) {   // negative: round the magnitude up
        uint32_t m = b & 0x7fffffffu;
        m = (m + 0xFFu) & ~0xFFu;
        return m | 0x80000000u;
    }
    return b & ~0xFFu;
}

// smallest biased exponent e (quantum 2^(e-127)) with origin + 254 quanta >= hi
__device__ __forceinline__ uint32_t pick_exp_w(float origin, float hi)
{
    float ext = hi - origin;
    uint32_t e = 1;
    if (ext > 0.f) {
        int ex;
        frexpf(ext / 255.0f, &ex);
        e = (uint32_t)max(1, min(254, ex + 127 - 1));
    }
    while (e < 254 && __fmaf_rn(254.0f, __uint_as_float(e << 23), origin) < hi) ++e;
    return e;
}

// outward-rounded quantised bounds with one quantum of padding on each side
__device__ __forceinline__ void quant_w(float lo, float hi, float o, float sc, uint32_t &qlo, uint32_t &qhi)
{
    float a = floorf(__fdiv_rd(__fsub_rd(lo, o), sc));
    float b = ceilf(__fdiv_ru(__fsub_ru(hi, o), sc));
    int ql = (int)fmaxf(0.f, fminf(255.f, a));
    int qh = (int)fmaxf(0.f, fminf(255.f, b));
    while (ql > 0 && __fmaf_rn((float)ql, sc, o) > lo) --ql;
    while (qh < 255 && __fmaf_rn((float)qh, sc, o) < hi) ++qh;
    qlo = (uint32_t)max(0, ql - 1);
    qhi = (uint32_t)min(255, qh + 1);
}

__device__ __forceinline__ float area_of(float3 lo, float3 hi)
{
    float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    return dx * dy + dy * dz + dz * dx;
}

// box of a leaf's primitives (the root of a scene no larger than one leaf)
__device__ void leaf_box(const float4 *prims, int32_t ref, float3 &lo, float3 &hi)
{
    lo = make_float3(INFINITY, INFINITY, INFINITY);
    hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    uint32_t first = leaf_first(ref), cnt = leaf_count(ref);
    for (uint32_t k = 0; k < cnt; ++k) {
        const float4 *p = prims + 3 * (size_t)(first + k);
        float4 a = p[0], b = p[1], c = p[2];
        if (__float_as_uint(a.w) & SPHERE_BIT) {
            lo = make_float3(fminf(lo.x, __fsub_rd(a.x, b.x)), fminf(lo.y, __fsub_rd(a.y, b.x)),
                             fminf(lo.z, __fsub_rd(a.z, b.x)));
            hi = make_float3(fmaxf(hi.x, __fadd_ru(a.x, b.x)), fmaxf(hi.y, __fadd_ru(a.y, b.x)),
                             fmaxf(hi.z, __fadd_ru(a.z, b.x)));
        } else {
            lo = make_float3(fminf(lo.x, fminf(a.x, fminf(b.x, c.x))), fminf(lo.y, fminf(a.y, fminf(b.y, c.y))),
                             fminf(lo.z, fminf(a.z, fminf(b.z, c.z))));
            hi = make_float3(fmaxf(hi.x, fmaxf(a.x, fmaxf(b.x, c.x))), fmaxf(hi.y, fmaxf(a.y, fmaxf(b.y, c.y))),
                             fmaxf(hi.z, fmaxf(a.z, fmaxf(b.z, c.z))));
        }
    }
}

// child c (0 or 1) of binary node i: its ref and box
__device__ __forceinline__ void bin_child(const float4 *nodes, int32_t i, int c, int32_t &ref, float3 &lo, float3 &hi)
{
    const float4 *p = nodes + 4 * (size_t)i;
    float4 a = p[c], z = p[2], d = p[3];
    lo = make_float3(a.x, a.z, c == 0 ? z.x : z.z);
    hi = make_float3(a.y, a.w, c == 0 ? z.y : z.w);
    ref = __float_as_int(c == 0 ? d.x : d.y);
}

// One wide node per thread.  ctr[0]: wide nodes allocated, ctr[1]: leaf
// primitives placed, ctr[2]: items of the next level, ctr[3]: error flag.
__global__ void k_wide_level(const float4 *__restrict__ bnodes, const float4 *__restrict__ bprims,
                             const WideItem *__restrict__ items, int nitems, WideItem *__restrict__ next,
                             int max_nodes, uint4 *__restrict__ wnodes, float4 *__restrict__ wprims, int n_prims,
                             int *ctr)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nitems) return;
    const WideItem W = items[it];
    int32_t cref[8];
    float3 clo[8], chi[8];
    int n = 0;
    if (W.bref >= 0) {
        bin_child(bnodes, W.bref, 0, cref[0], clo[0], chi[0]);
        bin_child(bnodes, W.bref, 1, cref[1], clo[1], chi[1]);
        n = 2;
        // open the largest internal child until 8 children or only leaves
        while (n < 8) {
            int best = -1;
            float ba = -1.f;
            for (int k = 0; k < n; ++k)
                if (cref[k] >= 0) {
                    float a = area_of(clo[k], chi[k]);
                    if (a > ba) {
                        ba = a;
                        best = k;
                    }
                }
            if (best < 0) break;
            const int32_t b = cref[best];
            bin_child(bnodes, b, 0, cref[best], clo[best], chi[best]);
            bin_child(bnodes, b, 1, cref[n], clo[n], chi[n]);
            ++n;
        }
    } else {
        cref[0] = W.bref;
        leaf_box(bprims, W.bref, clo[0], chi[0]);
        n = 1;
    }
    // drop empty leaves
    int m = 0;
    for (int k = 0; k < n; ++k)
        if (cref[k] != EMPTY_REF) {
            cref[m] = cref[k];
            clo[m] = clo[k];
            chi[m] = chi[k];
            ++m;
        }
    n = m;
    // node box and centre
    float3 lo = make_float3(INFINITY, INFINITY, INFINITY), hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    for (int k = 0; k < n; ++k) {
        lo = make_float3(fminf(lo.x, clo[k].x), fminf(lo.y, clo[k].y), fminf(lo.z, clo[k].z));
        hi = make_float3(fmaxf(hi.x, chi[k].x), fmaxf(hi.y, chi[k].y), fmaxf(hi.z, chi[k].z));
    }
    if (n == 0) lo = hi = make_float3(0.f, 0.f, 0.f);
    const float3 pc = make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
    // slots: greedily the (child, slot) pair whose centroid lies furthest
    // towards the slot's octant
    int slot_of[8], child_in[8];
    for (int s = 0; s < 8; ++s) child_in[s] = -1;
    for (int k = 0; k < n; ++k) slot_of[k] = -1;
    for (int round = 0; round < n; ++round) {
        float bv = -INFINITY;
        int bk = -1, bs = -1;
        for (int k = 0; k < n; ++k) {
            if (slot_of[k] >= 0) continue;
            const float3 c = make_float3(0.5f * (clo[k].x + chi[k].x) - pc.x, 0.5f * (clo[k].y + chi[k].y) - pc.y,
                                         0.5f * (clo[k].z + chi[k].z) - pc.z);
            for (int s = 0; s < 8; ++s) {
                if (child_in[s] >= 0) continue;
                float v = ((s & 1) ? c.x : -c.x) + ((s & 2) ? c.y : -c.y) + ((s & 4) ? c.z : -c.z);
                if (v > bv) {
                    bv = v;
                    bk = k;
                    bs = s;
                }
            }
        }
        slot_of[bk] = bs;
        child_in[bs] = bk;
    }
    // allocate internal children and leaf primitives
    int ni = 0, np = 0;
    uint32_t imask = 0;
    for (int s = 0; s < 8; ++s) {
        int k = child_in[s];
        if (k < 0) continue;
        if (cref[k] >= 0) {
            imask |= 1u << s;
            ++ni;
        } else {
            np += (int)leaf_count(cref[k]);
        }
    }
    const int child_base = ni ? atomicAdd(&ctr[0], ni) : 0;
    const int prim_base = np ? atomicAdd(&ctr[1], np) : 0;
    if (child_base + ni > max_nodes || prim_base + np > n_prims) {
        atomicExch(&ctr[3], 1);   // cannot happen for a valid binary tree
        return;
    }
    // node
    uint32_t ob[3], ex[3];
    float o[3], sc[3];
    const float alo[3] = {lo.x, lo.y, lo.z}, ahi[3] = {hi.x, hi.y, hi.z};
    for (int a = 0; a < 3; ++a) {
        ob[a] = origin_bits_w(alo[a]);
        o[a] = __uint_as_float(ob[a]);
        ex[a] = pick_exp_w(o[a], ahi[a]);
        sc[a] = __uint_as_float(ex[a] << 23);
    }
    uint32_t qlo[3][8], qhi[3][8], meta[8];
    int rank = 0, off = 0;
    for (int s = 0; s < 8; ++s) {
        int k = child_in[s];
        meta[s] = 0;
        if (k < 0) {
            for (int a = 0; a < 3; ++a) {
                qlo[a][s] = 255;
                qhi[a][s] = 0;
            }
            continue;
        }
        const float cl[3] = {clo[k].x, clo[k].y, clo[k].z}, ch[3] = {chi[k].x, chi[k].y, chi[k].z};
        for (int a = 0; a < 3; ++a) quant_w(cl[a], ch[a], o[a], sc[a], qlo[a][s], qhi[a][s]);
        if (cref[k] >= 0) {
            int slot_next = atomicAdd(&ctr[2], 1);
            next[slot_next] = WideItem{cref[k], child_base + rank};
            ++rank;
        } else {
            const uint32_t first = leaf_first(cref[k]), cnt = leaf_count(cref[k]);
            meta[s] = (cnt << 5) | (uint32_t)off;
            for (uint32_t j = 0; j < cnt; ++j) {
                const float4 *src = bprims + 3 * (size_t)(first + j);
                float4 *dst = wprims + 3 * (size_t)(prim_base + off + (int)j);
                dst[0] = src[0];
                dst[1] = src[1];
                dst[2] = src[2];
            }
            off += (int)cnt;
        }
    }
    uint4 *w = wnodes + 5 * (size_t)W.widx;
    w[0] = make_uint4(ob[0] | ex[0], ob[1] | ex[1], ob[2] | ex[2], imask);
    w[1] = make_uint4((uint32_t)child_base, (uint32_t)prim_base,
                      meta[0] | (meta[1] << 8) | (meta[2] << 16) | (meta[3] << 24),
                      meta[4] | (meta[5] << 8) | (meta[6] << 16) | (meta[7] << 24));
    uint32_t q[12];
    for (int a = 0; a < 3; ++a) {
        q[2 * a] = qlo[a][0] | (qlo[a][1] << 8) | (qlo[a][2] << 16) | (qlo[a][3] << 24);
        q[2 * a + 1] = qlo[a][4] | (qlo[a][5] << 8) | (qlo[a][6] << 16) | (qlo[a][7] << 24);
        q[6 + 2 * a] = qhi[a][0] | (qhi[a][1] << 8) | (qhi[a][2] << 16) | (qhi[a][3] << 24);
        q[6 + 2 * a + 1] = qhi[a][4] | (qhi[a][5] << 8) | (qhi[a][6] << 16) | (qhi[a][7] << 24);
    }
    w[2] = make_uint4(q[0], q[1], q[2], q[3]);
    w[3] = make_uint4(q[4], q[5], q[6], q[7]);
    w[4] = make_uint4(q[8], q[9], q[10], q[11]);
}

}  // namespace

xtgpu_status build_wide(xtgpu_scene *sc, cudaStream_t s)
{
    DevScene &S = sc->dev;
    const int n = (int)sc->n_prims;
    if (sc->leaf_size > WIDE_MAX_LEAF) {
        set_error("xtgpu_bvh_build: the 8-wide format takes leaves of at most 3 primitives");
        return XTGPU_ERR_INVALID;
    }
    dfree(sc->nodesW);
    dfree(sc->leafW);
    sc->builtW = false;
    sc->depthW = 0;
    sc->n_wide = 0;
    if (n == 0) {
        S.nodesW = nullptr;
        S.leafW = nullptr;
        S.rootW = -1;
        sc->builtW = true;
        return XTGPU_OK;
    }
    // every wide node starts from a distinct binary internal node (or the root leaf)
    const int max_nodes = std::max(1, n - 1);
    XTG_TRY(dalloc(sc->nodesW, sizeof(uint4) * 5 * (size_t)max_nodes, s));
    XTG_TRY(dalloc(sc->leafW, sizeof(float4) * 3 * (size_t)n, s));
    HostBuf itemsA, itemsB, ctrb;
    XTG_TRY(dalloc(itemsA, sizeof(WideItem) * (size_t)max_nodes, s));
    XTG_TRY(dalloc(itemsB, sizeof(WideItem) * (size_t)max_nodes, s));
    XTG_TRY(dalloc(ctrb, sizeof(int) * 4, s));
    int *ctr = (int *)ctrb.p;
    WideItem root{S.root, 0};
    int hctr[4] = {1, 0, 0, 0};
    XTG_CUDA(cudaMemcpyAsync(itemsA.p, &root, sizeof(root), cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(ctr, hctr, sizeof(hctr), cudaMemcpyHostToDevice, s));
    WideItem *cur = (WideItem *)itemsA.p, *nxt = (WideItem *)itemsB.p;
    int nitems = 1, levels = 0;
    xtgpu_status st = XTGPU_OK;
    while (nitems > 0) {
        if (++levels > 128) {   // a binary tree of depth <= 64 cannot give more levels
            set_error("xtgpu_bvh_build: wide collapse did not terminate");
            st = XTGPU_ERR_CUDA;
            break;
        }
        k_wide_level<<<(nitems + 127) / 128, 128, 0, s>>>(S.nodes32, S.leaf_prims, cur, nitems, nxt, max_nodes,
                                                           (uint4 *)sc->nodesW.p, (float4 *)sc->leafW.p, n, ctr);
        int back[4];
        cudaError_t e = cudaMemcpyAsync(back, ctr, sizeof(back), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "wide collapse", __FILE__, __LINE__);
            break;
        }
        if (back[3]) {
            set_error("xtgpu_bvh_build: wide collapse overflow");
            st = XTGPU_ERR_CUDA;
            break;
        }
        nitems = back[2];
        sc->n_wide = back[0];
        int zero = 0;
        e = cudaMemcpyAsync(ctr + 2, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "wide collapse", __FILE__, __LINE__);
            break;
        }
        std::swap(cur, nxt);
    }
    dfree(itemsA);
    dfree(itemsB);
    dfree(ctrb);
    if (st != XTGPU_OK) {
        dfree(sc->nodesW);
        dfree(sc->leafW);
        return st;
    }
    sc->depthW = levels;
    S.nodesW = (const uint4 *)sc->nodesW.p;
    S.leafW = (const float4 *)sc->leafW.p;
    S.rootW = 0;
    sc->builtW = true;
    return XTGPU_OK;
}

}  // namespace xtg
