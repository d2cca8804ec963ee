// 8-wide BVH with 8-bit quantised child bounds, collapsed from the binary LBVH
// on the device.  The node layout, the traversal order and the cost-optimal
// collapse follow Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal
// on GPUs Through Compressed Wide BVHs" (HPG 2017).
//
// Which binary nodes become wide nodes, and which subtrees become leaves, is
// chosen one of two ways (xtgpu_tuning::wide_collapse):
//   * 1, cost-optimal (default): a bottom-up dynamic programme over the binary
//     tree (k_wide_dp) gives every node n and budget i = 1..7 the lowest
//     surface-area cost C(n, i) of representing n's subtree by at most i
//     children of a wide node.  C(n, 1) is the cheaper of one leaf (at most 3
//     primitives: A(n) * c_prim * P(n)) and one internal wide node (A(n) *
//     c_node + the best split of 8 children between n's two binary
//     children); C(n, i > 1) is the better of C(n, i - 1) and the best split of
//     i between the two children.  The emission follows the recorded choices;
//   * 0, greedy: a wide node repeatedly opens the internal child with the
//     largest surface area until it has 8 children or only leaves are left,
//     and every binary leaf is one wide leaf.
//
// Build, one kernel launch per level of the wide tree (top down):
//   * a wide node starts from one binary internal node and takes its children
//     as above;
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

// --- cost-optimal collapse --------------------------------------------------
// Per binary internal node: C(n, i) for i = 1..7, the left child's share k of
// the best split of j = 2..8 children, which C(n, i) come from a split (bit
// i - 1, i >= 2) and whether C(n, 1) is a leaf (bit 7), and P(n).
struct WideDP {
    float c[7];
    uint8_t split[7];
    uint8_t use;
    int32_t prims;
};

constexpr float WIDE_NODE_COST = 1.0f;

__device__ __forceinline__ float3 fmin3(float3 a, float3 b)
{
    return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z));
}
__device__ __forceinline__ float3 fmax3(float3 a, float3 b)
{
    return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z));
}

__global__ void k_wide_parents(int ni, const float4 *__restrict__ bnodes, int32_t *__restrict__ parent)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ni) return;
    const float4 d = bnodes[4 * (size_t)n + 3];
    const int32_t c0 = __float_as_int(d.x), c1 = __float_as_int(d.y);
    if (c0 >= 0 && c0 < ni) parent[c0] = n;
    if (c1 >= 0 && c1 < ni) parent[c1] = n;
}

// the DP entry of binary node n from its children's (computed before)
__device__ void wide_dp_node(const float4 *__restrict__ bnodes, WideDP *dp, int32_t n, float cprim)
{
    float ck[2][7];
    int32_t pk[2];
    float3 lo = make_float3(INFINITY, INFINITY, INFINITY), hi = make_float3(-INFINITY, -INFINITY, -INFINITY);
    for (int c = 0; c < 2; ++c) {
        int32_t ref;
        float3 cl, ch;
        bin_child(bnodes, n, c, ref, cl, ch);
        lo = fmin3(lo, cl);
        hi = fmax3(hi, ch);
        if (ref >= 0) {
            // written by another thread before its fence: read past L1
            const float *src = (const float *)(dp + ref);
            for (int i = 0; i < 7; ++i) ck[c][i] = __ldcg(src + i);
            pk[c] = __ldcg(&dp[ref].prims);
        } else {
            const int cnt = (int)leaf_count(ref);
            const float v = ref == EMPTY_REF ? 0.f : area_of(cl, ch) * cprim * (float)cnt;
            for (int i = 0; i < 7; ++i) ck[c][i] = v;
            pk[c] = cnt;
        }
    }
    WideDP out;
    out.prims = pk[0] + pk[1];
    float dist[9];
    for (int j = 2; j <= 8; ++j) {
        float best = INFINITY;
        int bk = 1;
        for (int k = 1; k < j; ++k) {
            const float v = ck[0][k - 1] + ck[1][j - k - 1];
            if (v < best) {
                best = v;
                bk = k;
            }
        }
        dist[j] = best;
        out.split[j - 2] = (uint8_t)bk;
    }
    const float A = area_of(lo, hi);
    const float cleaf = out.prims <= WIDE_MAX_LEAF ? A * cprim * (float)out.prims : INFINITY;
    const float cint = A * WIDE_NODE_COST + dist[8];
    out.use = 0;
    out.c[0] = fminf(cleaf, cint);
    if (cleaf <= cint) out.use |= 0x80u;
    for (int i = 2; i <= 7; ++i) {
        if (dist[i] < out.c[i - 2]) {
            out.c[i - 1] = dist[i];
            out.use |= (uint8_t)(1u << (i - 1));
        } else {
            out.c[i - 1] = out.c[i - 2];
        }
    }
    dp[n] = out;
}

// Bottom up: a thread starts at every node without internal children and
// climbs while it is the last of a node's internal children to finish.
__global__ void k_wide_dp(int ni, const float4 *__restrict__ bnodes, const int32_t *__restrict__ parent,
                          unsigned *__restrict__ arrived, WideDP *dp, float cprim, int *err)
{
    int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ni) return;
    {
        const float4 d = bnodes[4 * (size_t)n + 3];
        if (__float_as_int(d.x) >= 0 || __float_as_int(d.y) >= 0) return;
    }
    for (int guard = 0;; ++guard) {
        if (guard > 256) {   // deeper than any tree this build makes: report, never loop forever
            atomicExch(err, 1);
            return;
        }
        wide_dp_node(bnodes, dp, n, cprim);
        __threadfence();
        const int32_t p = parent[n];
        if (p < 0) return;
        const float4 d = bnodes[4 * (size_t)p + 3];
        const unsigned need = (__float_as_int(d.x) >= 0 ? 1u : 0u) + (__float_as_int(d.y) >= 0 ? 1u : 0u);
        if (atomicAdd(&arrived[p], 1u) + 1u < need) return;
        __threadfence();
        n = p;
    }
}

// The children of the wide node made from binary node `root` under the DP's
// choices: up to 8 (ref, box) pairs; a subtree chosen as a leaf becomes the
// leaf ref of its primitives (contiguous in the leaf order).
__device__ int wide_children_dp(const float4 *__restrict__ bnodes, const WideDP *__restrict__ dp, int32_t root,
                                int32_t cref[8], float3 clo[8], float3 chi[8])
{
    int32_t sref[16];
    int sb[16];
    float3 slo[16], shi[16];
    int sp = 0, n = 0;
    const int k8 = dp[root].split[8 - 2];
    bin_child(bnodes, root, 1, sref[sp], slo[sp], shi[sp]);
    sb[sp++] = 8 - k8;
    bin_child(bnodes, root, 0, sref[sp], slo[sp], shi[sp]);
    sb[sp++] = k8;
    while (sp > 0 && n < 8) {
        --sp;
        const int32_t ref = sref[sp];
        int i = sb[sp];
        const float3 lo = slo[sp], hi = shi[sp];
        if (ref < 0) {
            cref[n] = ref;
            clo[n] = lo;
            chi[n] = hi;
            ++n;
            continue;
        }
        const WideDP &D = dp[ref];
        while (i > 1 && !(D.use & (1u << (i - 1)))) --i;
        if (i == 1) {
            int32_t r = ref;
            if (D.use & 0x80u)
                for (int g = 0; r >= 0 && g < 64; ++g) r = __float_as_int(bnodes[4 * (size_t)r + 3].x);
            // the subtree's primitives start at its leftmost leaf; a walk that
            // ends on no leaf (a malformed tree) keeps the node internal
            cref[n] = (D.use & 0x80u) && r < 0 && r != EMPTY_REF ? leaf_ref(leaf_first(r), (uint32_t)D.prims) : ref;
            clo[n] = lo;
            chi[n] = hi;
            ++n;
            continue;
        }
        if (sp + 2 > 16) break;   // budgets sum to at most 8: cannot happen
        const int k = D.split[i - 2];
        bin_child(bnodes, ref, 1, sref[sp], slo[sp], shi[sp]);
        sb[sp++] = i - k;
        bin_child(bnodes, ref, 0, sref[sp], slo[sp], shi[sp]);
        sb[sp++] = k;
    }
    return n;
}

// One wide node per thread.  ctr[0]: wide nodes allocated, ctr[1]: leaf
// primitives placed, ctr[2]: items of the next level, ctr[3]: error flag.
__global__ void k_wide_level(const float4 *__restrict__ bnodes, const float4 *__restrict__ bprims,
                             const WideDP *__restrict__ dp, const WideItem *__restrict__ items, int nitems,
                             WideItem *__restrict__ next, int max_nodes, uint4 *__restrict__ wnodes,
                             float4 *__restrict__ wprims, int n_prims, int *ctr)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nitems) return;
    const WideItem W = items[it];
    int32_t cref[8];
    float3 clo[8], chi[8];
    int n = 0;
    if (W.bref >= 0 && dp) {
        n = wide_children_dp(bnodes, dp, W.bref, cref, clo, chi);
    } else if (W.bref >= 0) {
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
    const xtgpu_tuning &T = scene_tuning(sc);
    const int ni = n - 1;
    HostBuf dpb;
    if (T.wide_collapse == 1 && ni > 0 && S.root >= 0) {
        // the cost tables, bottom up
        HostBuf parb, arrb, errb;
        XTG_TRY(dalloc(dpb, sizeof(WideDP) * (size_t)ni, s));
        XTG_TRY(dalloc(parb, sizeof(int32_t) * (size_t)ni, s));
        XTG_TRY(dalloc(arrb, sizeof(unsigned) * (size_t)ni, s));
        XTG_TRY(dalloc(errb, sizeof(int), s));
        XTG_CUDA(cudaMemsetAsync(parb.p, 0xff, sizeof(int32_t) * (size_t)ni, s));
        XTG_CUDA(cudaMemsetAsync(arrb.p, 0, sizeof(unsigned) * (size_t)ni, s));
        XTG_CUDA(cudaMemsetAsync(errb.p, 0, sizeof(int), s));
        k_wide_parents<<<(ni + 255) / 256, 256, 0, s>>>(ni, S.nodes32, (int32_t *)parb.p);
        const float cprim = T.wide_prim_cost > 0.f ? T.wide_prim_cost : 1.0f;
        k_wide_dp<<<(ni + 127) / 128, 128, 0, s>>>(ni, S.nodes32, (const int32_t *)parb.p, (unsigned *)arrb.p,
                                                   (WideDP *)dpb.p, cprim, (int *)errb.p);
        int err = 0;
        cudaError_t e = cudaMemcpyAsync(&err, errb.p, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        dfree(parb);
        dfree(arrb);
        dfree(errb);
        if (e != cudaSuccess) {
            dfree(dpb);
            return cuda_fail(e, "wide collapse costs", __FILE__, __LINE__);
        }
        if (err) {
            dfree(dpb);
            set_error("xtgpu_bvh_build: wide collapse costs did not reach the root");
            return XTGPU_ERR_CUDA;
        }
    }
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
        k_wide_level<<<(nitems + 127) / 128, 128, 0, s>>>(S.nodes32, S.leaf_prims, (const WideDP *)dpb.p, cur,
                                                           nitems, nxt, max_nodes, (uint4 *)sc->nodesW.p,
                                                           (float4 *)sc->leafW.p, n, ctr);
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
    dfree(dpb);
    if (st != XTGPU_OK) {
        dfree(sc->nodesW);
        dfree(sc->leafW);
        return st;
    }
    sc->depthW = levels;
    sc->wide_collapse = T.wide_collapse;
    sc->wide_prim_cost = T.wide_prim_cost;
    S.nodesW = (const uint4 *)sc->nodesW.p;
    S.leafW = (const float4 *)sc->leafW.p;
    S.rootW = 0;
    sc->builtW = true;
    return XTGPU_OK;
}

}  // namespace xtg
