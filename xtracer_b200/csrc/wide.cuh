// Closest-hit traversal of the 8-wide quantised BVH built by wide.cu.
//
// A node visit tests its 8 child boxes in quantised space (one FMA per bound:
// t(q) = q * (2^e * inv) + (origin - ray.o) * inv), tests the primitives of
// every hit leaf child at once, and goes on with the nearest hit internal
// child.  The other hit internal children stay behind as one stack entry (node
// group): the base index, the node's internal-child mask and the hit children
// as bits in visiting order.  Visiting order is slot ^ m, m the ray's sign
// bits, which takes the children on the ray's entry side first (the build
// puts children in slots by direction).  Ylitie, Karras and Laine, HPG 2017.
#pragma once

#include "traverse.cuh"

namespace xtg {

constexpr int WIDE_MAX_LEAF = 3;

// far-distance scale of the quantised box test (as for the binary Q8 nodes)
#define XTG_TFAR_SCALE_W8 1.0000015f

__device__ __forceinline__ float q8(uint32_t w, int k) { return (float)((w >> (8 * k)) & 0xFFu); }

// Ray sign bits: bit k set if direction component k is negative.
__device__ __forceinline__ uint32_t ray_octant(const RayPre &r)
{
    return (r.d.x < 0.f ? 1u : 0u) | (r.d.y < 0.f ? 2u : 0u) | (r.d.z < 0.f ? 4u : 0u);
}

// One step: visits `node`, tests its hit leaf primitives and sets `node` to
// the next node to visit.  Returns true when the traversal is over (nothing
// left on the stack, or the stack overflowed).
template <int STACK>
__device__ __forceinline__ bool wide_step(const SceneView &V, const RayPre &r, uint32_t m, float tmin, float &tmax,
                                          uint32_t &prim, float &bu, float &bv, int32_t &node, int &sp,
                                          uint2 *stack, int32_t *ctl_overflow, uint32_t &nv, uint32_t &np)
{
    const uint4 *p = (const uint4 *)V.nodes + 5 * (size_t)node;
    const uint4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3), w4 = __ldg(p + 4);
    ++nv;
    const float sx = __uint_as_float((w0.x & 0xFFu) << 23) * r.inv.x;
    const float sy = __uint_as_float((w0.y & 0xFFu) << 23) * r.inv.y;
    const float sz = __uint_as_float((w0.z & 0xFFu) << 23) * r.inv.z;
    const float bx = fmaf(__uint_as_float(w0.x & ~0xFFu), r.inv.x, -r.oinv.x);
    const float by = fmaf(__uint_as_float(w0.y & ~0xFFu), r.inv.y, -r.oinv.y);
    const float bz = fmaf(__uint_as_float(w0.z & ~0xFFu), r.inv.z, -r.oinv.z);
    const uint32_t imask = w0.w;
    const uint32_t meta[2] = {w1.z, w1.w};
    // qlo.x w2.x,w2.y  qlo.y w2.z,w2.w  qlo.z w3.x,w3.y  qhi.x w3.z,w3.w  qhi.y w4.x,w4.y  qhi.z w4.z,w4.w
    const uint32_t lx[2] = {w2.x, w2.y}, ly[2] = {w2.z, w2.w}, lz[2] = {w3.x, w3.y};
    const uint32_t hx[2] = {w3.z, w3.w}, hy[2] = {w4.x, w4.y}, hz[2] = {w4.z, w4.w};
    uint32_t hits = 0, leaves = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int h = s >> 2, k = s & 3;
        const uint32_t mb = (meta[h] >> (8 * k)) & 0xFFu;
        const bool inner = (imask >> s) & 1u;
        if (!inner && mb == 0u) continue;   // unused slot
        const float tx0 = fmaf(q8(lx[h], k), sx, bx), tx1 = fmaf(q8(hx[h], k), sx, bx);
        const float ty0 = fmaf(q8(ly[h], k), sy, by), ty1 = fmaf(q8(hy[h], k), sy, by);
        const float tz0 = fmaf(q8(lz[h], k), sz, bz), tz1 = fmaf(q8(hz[h], k), sz, bz);
        float tn;
        if (!slab_t(tx0, tx1, ty0, ty1, tz0, tz1, tmin, tmax, XTG_TFAR_SCALE_W8, tn)) continue;
        if (inner) hits |= 1u << (s ^ m);
        else leaves |= ((1u << (mb >> 5)) - 1u) << (mb & 31u);
    }
    // primitives of the hit leaf children
    const uint32_t pbase = w1.y;
    while (leaves) {
        const int k = __ffs(leaves) - 1;
        leaves &= leaves - 1u;
        ++np;
        prim_test(V.leaf, pbase + (uint32_t)k, r, tmin, tmax, prim, bu, bv);
    }
    uint32_t base = w1.x, im = imask;
    if (!hits) {
        // next node group from the stack
        if (sp == 0) return true;
        const uint2 e = stack[--sp];
        base = e.x;
        im = e.y & 0xFFu;
        hits = e.y >> 8;
    }
    const int key = __ffs(hits) - 1;
    hits &= hits - 1u;
    const uint32_t slot = (uint32_t)key ^ m;
    node = (int32_t)(base + (uint32_t)__popc(im & ((1u << slot) - 1u)));
    if (hits) {
        if (sp >= STACK) {
            *ctl_overflow = 1;
            return true;
        }
        stack[sp++] = make_uint2(base, im | (hits << 8));
    }
    return false;
}

template <int STACK>
__device__ __forceinline__ void trace_wide(const SceneView &V, const RayPre &r, float tmin, float &tmax,
                                           uint32_t &prim, float &bu, float &bv, int32_t *ctl_overflow, uint32_t &nv,
                                           uint32_t &np)
{
    const uint32_t m = ray_octant(r);
    uint2 stack[STACK];
    int sp = 0;
    int32_t node = V.root;
    if (node >= 0)
        for (uint32_t guard = 0;; ++guard) {
            if (guard >= (1u << 22)) {   // corrupted tree: report, never loop forever
                *ctl_overflow = 1;
                break;
            }
            if (wide_step<STACK>(V, r, m, tmin, tmax, prim, bu, bv, node, sp, stack, ctl_overflow, nv, np)) break;
        }
    for (int p = 0; p < V.n_planes; ++p)
        if (hit_plane(r, __ldg(V.planes + p), tmin, tmax)) {
            prim = V.plane_base + (uint32_t)p;
            bu = bv = 0.f;
        }
}

}  // namespace xtg
