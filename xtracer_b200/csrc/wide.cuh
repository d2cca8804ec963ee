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

// Ray sign bits: bit k set if component k of the (clamped) inverse direction
// is negative; a zero component counts by the sign of its clamped inverse.
__device__ __forceinline__ uint32_t ray_octant(const RayPre &r)
{
    return (r.inv.x < 0.f ? 1u : 0u) | (r.inv.y < 0.f ? 2u : 0u) | (r.inv.z < 0.f ? 4u : 0u);
}

// Bit s of x moved to bit s ^ m (8 bits).
__device__ __forceinline__ uint32_t permute_xor8(uint32_t x, uint32_t m)
{
    if (m & 1u) x = ((x & 0x55u) << 1) | ((x >> 1) & 0x55u);
    if (m & 2u) x = ((x & 0x33u) << 2) | ((x >> 2) & 0x33u);
    if (m & 4u) x = ((x & 0x0Fu) << 4) | ((x >> 4) & 0x0Fu);
    return x;
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
    const uint4 w0 = __ldg(p), w1 = __ldg(p + 1);
    // the stack's top entry, read with the node so that a pop at the end of
    // the step does not wait for local memory (entry 0, unused, when empty)
    const uint2 top = stack[sp > 0 ? sp - 1 : 0];
    ++nv;
    const float sx = __uint_as_float((w0.x & 0xFFu) << 23) * r.inv.x;
    const float sy = __uint_as_float((w0.y & 0xFFu) << 23) * r.inv.y;
    const float sz = __uint_as_float((w0.z & 0xFFu) << 23) * r.inv.z;
    const float bx = fmaf(__uint_as_float(w0.x & ~0xFFu), r.inv.x, -r.oinv.x);
    const float by = fmaf(__uint_as_float(w0.y & ~0xFFu), r.inv.y, -r.oinv.y);
    const float bz = fmaf(__uint_as_float(w0.z & ~0xFFu), r.inv.z, -r.oinv.z);
    const uint32_t imask = w0.w;
    // bound words, 4 slots each: qlo.x at word 8+h, qlo.y 10+h, qlo.z 12+h,
    // qhi.x 14+h, qhi.y 16+h, qhi.z 18+h (h = 0 for slots 0-3, 1 for 4-7).
    // Both halves unrolled, so the second half's loads are issued with the
    // first's instead of after it (a few spilled words, cheaper than the
    // second wait).  The near plane of an axis is its lower bound when the ray
    // goes up that axis, else the upper one, so each bound takes one FMA and
    // no swap.  An unused slot (qlo 255 > qhi 0) is behind its own far plane
    // and never hits.
    const uint32_t *qw = (const uint32_t *)(p + 2);
    uint32_t hitbits = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t lx = __ldg(qw + h), ly = __ldg(qw + 2 + h), lz = __ldg(qw + 4 + h);
        const uint32_t hx = __ldg(qw + 6 + h), hy = __ldg(qw + 8 + h), hz = __ldg(qw + 10 + h);
        const uint32_t nx = (m & 1u) ? hx : lx, fx = (m & 1u) ? lx : hx;
        const uint32_t ny = (m & 2u) ? hy : ly, fy = (m & 2u) ? ly : hy;
        const uint32_t nz = (m & 4u) ? hz : lz, fz = (m & 4u) ? lz : hz;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float tn = fmaxf(fmaxf(fmaf(q8(nx, k), sx, bx), fmaf(q8(ny, k), sy, by)),
                                   fmaxf(fmaf(q8(nz, k), sz, bz), tmin));
            const float tf = fminf(fminf(fmaf(q8(fx, k), sx, bx), fmaf(q8(fy, k), sy, by)),
                                   fminf(fmaf(q8(fz, k), sz, bz), tmax));
            hitbits |= (tn <= tf * XTG_TFAR_SCALE_W8 ? 1u : 0u) << (4 * h + k);
        }
    }
    uint32_t hits = permute_xor8(hitbits & imask, m);
    uint32_t leaves = 0;
    for (uint32_t lh = hitbits & ~imask; lh; lh &= lh - 1u) {
        const int slot = __ffs(lh) - 1;
        const uint32_t mb = ((slot < 4 ? w1.z : w1.w) >> (8 * (slot & 3))) & 0xFFu;
        leaves |= ((1u << (mb >> 5)) - 1u) << (mb & 31u);
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
        --sp;
        const uint2 e = top;
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
    stack[0] = make_uint2(0u, 0u);   // wide_step reads entry 0 ahead even when the stack is empty
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
