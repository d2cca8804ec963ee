// Ray traversal device code: closest hit over the scene's BVH (triangles and
// spheres) plus the scene's infinite planes, which no BVH can bound.
//
// Semantics follow Scene::intersection (src/xtcore/scene.cc:191-216): the
// nearest hit over every surface; spheres are hit only from outside
// (t = min(t1, t2) must be positive, math/sphere.cc:35-62), planes and
// triangles from both sides (math/plane.cc:19-61, math/triangle.cc:82-123).
//
// Triangles use the watertight test of Woop, Benthin and Wald ("Watertight
// Ray/Triangle Intersection", JCGT 2013) in FP32: shear into ray space, 2D
// edge functions with the products rounded separately (no FMA contraction, so
// a shared edge gives exactly opposite values in both triangles) and an FP64
// re-evaluation when an edge function is exactly zero.  Box tests are the slab
// test with the far distance scaled up by 1 + 2*gamma(3) (Ize, "Robust BVH Ray
// Traversal", JCGT 2013) so rounding never culls a box the ray touches.
#pragma once

#include "xtgpu_internal.cuh"

namespace xtg {

struct RayPre {
    float3 o, d, inv, oinv;
    int kx, ky, kz;
    float Sx, Sy, Sz;
};

__device__ __forceinline__ float comp(const float3 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ void ray_pre(float3 o, float3 d, RayPre &r)
{
    r.o = o;
    r.d = d;
    const float tiny = 1e-20f;
    float dx = fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x;
    float dy = fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y;
    float dz = fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z;
    r.inv = make_float3(1.0f / dx, 1.0f / dy, 1.0f / dz);
    r.oinv = make_float3(o.x * r.inv.x, o.y * r.inv.y, o.z * r.inv.z);
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    float dk = comp(d, kz);
    if (dk < 0.f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.Sx = comp(d, kx) / dk;
    r.Sy = comp(d, ky) / dk;
    r.Sz = 1.0f / dk;
}

// 1 + 2*gamma(3) rounded up
#define XTG_TFAR_SCALE 1.00000072f

__device__ __forceinline__ bool slab(const RayPre &r, float lx, float hx, float ly, float hy, float lz, float hz,
                                     float tmin, float tmax, float &tnear)
{
    float tx0 = fmaf(lx, r.inv.x, -r.oinv.x), tx1 = fmaf(hx, r.inv.x, -r.oinv.x);
    float ty0 = fmaf(ly, r.inv.y, -r.oinv.y), ty1 = fmaf(hy, r.inv.y, -r.oinv.y);
    float tz0 = fmaf(lz, r.inv.z, -r.oinv.z), tz1 = fmaf(hz, r.inv.z, -r.oinv.z);
    float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    tnear = tn;
    return tn <= tf * XTG_TFAR_SCALE;
}

// FP64 re-evaluation of the edge functions (the paper's fallback).
static __device__ __noinline__ void edges_fp64(float Ax, float Ay, float Bx, float By, float Cx, float Cy, float &U,
                                        float &V, float &W)
{
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
}

// Two-sided watertight triangle test.  On a hit inside (tmin, tmax) updates
// tmax and the barycentrics of v1 (u) and v2 (v).
// A hit replaces the current one if it is nearer, or as near and of a lower
// primitive id: the closest hit then does not depend on the order in which a
// traversal meets the primitives (binary or wide nodes, any child order).
__device__ __forceinline__ bool nearer(float t, float tmax, uint32_t id, uint32_t cur)
{
    return t < tmax || (t == tmax && cur != 0xffffffffu && id < cur);
}

__device__ __forceinline__ bool hit_triangle(const RayPre &r, float3 v0, float3 v1, float3 v2, float tmin,
                                             float &tmax, float &bu, float &bv, uint32_t id, uint32_t cur)
{
    float3 A = make_float3(v0.x - r.o.x, v0.y - r.o.y, v0.z - r.o.z);
    float3 B = make_float3(v1.x - r.o.x, v1.y - r.o.y, v1.z - r.o.z);
    float3 C = make_float3(v2.x - r.o.x, v2.y - r.o.y, v2.z - r.o.z);
    float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    float Ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.Sx, Akz));
    float Ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.Sy, Akz));
    float Bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.Sx, Bkz));
    float By = __fsub_rn(comp(B, r.ky), __fmul_rn(r.Sy, Bkz));
    float Cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.Sx, Ckz));
    float Cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.Sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.f || V == 0.f || W == 0.f) edges_fp64(Ax, Ay, Bx, By, Cx, Cy, U, V, W);
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    float det = U + V + W;
    if (det == 0.f) return false;
    float Az = r.Sz * Akz, Bz = r.Sz * Bkz, Cz = r.Sz * Ckz;
    float T = U * Az + V * Bz + W * Cz;
    float rcp = 1.0f / det;
    float t = T * rcp;
    if (!(t > tmin && nearer(t, tmax, id, cur))) return false;
    tmax = t;
    bu = V * rcp;
    bv = W * rcp;
    return true;
}

// Sphere hit only from outside: the nearer root must lie in (tmin, tmax).
// Discriminant in the form of Haines et al., "Precision Improvements for
// Ray/Sphere Intersection" (Ray Tracing Gems, 2019); unit direction assumed.
__device__ __forceinline__ bool hit_sphere(const RayPre &r, float3 c, float rad, float tmin, float &tmax, uint32_t id,
                                           uint32_t cur)
{
    float3 f = make_float3(r.o.x - c.x, r.o.y - c.y, r.o.z - c.z);
    float b = f.x * r.d.x + f.y * r.d.y + f.z * r.d.z;
    float3 h = make_float3(f.x - b * r.d.x, f.y - b * r.d.y, f.z - b * r.d.z);
    float r2 = rad * rad;
    float disc = r2 - (h.x * h.x + h.y * h.y + h.z * h.z);
    if (!(disc > 0.f)) return false;
    float cc = (f.x * f.x + f.y * f.y + f.z * f.z) - r2;
    float q = -b - copysignf(sqrtf(disc), b);
    float t0 = cc / q, t1 = q;
    float tn = fminf(t0, t1);
    if (!(tn > tmin && nearer(tn, tmax, id, cur))) return false;
    tmax = tn;
    return true;
}

// Infinite plane through |n| * offset (plane.cc:33-41), two-sided.
__device__ __forceinline__ bool hit_plane(const RayPre &r, float4 pl, float tmin, float &tmax)
{
    float ndd = pl.x * r.d.x + pl.y * r.d.y + pl.z * r.d.z;
    if (fabsf(ndd) < 1e-8f) return false;
    float3 v = make_float3(fabsf(pl.x) * pl.w - r.o.x, fabsf(pl.y) * pl.w - r.o.y, fabsf(pl.z) * pl.w - r.o.z);
    float t = (v.x * pl.x + v.y * pl.y + v.z * pl.z) / ndd;
    if (!(t > tmin && t < tmax)) return false;
    tmax = t;
    return true;
}

// Both children of a node: entry distances and whether each box is hit.
struct Pair {
    float t0, t1;
    bool h0, h1;
    int32_t c0, c1;
};

__device__ __forceinline__ bool slab_t(float tx0, float tx1, float ty0, float ty1, float tz0, float tz1, float tmin,
                                       float tmax, float scale, float &tnear)
{
    float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    tnear = tn;
    return tn <= tf * scale;
}

template <int FMT>
__device__ __forceinline__ void node_pair(const void *nodes, int32_t i, const RayPre &r, float tmin, float tmax,
                                          Pair &P);

// 64-byte node: (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y) (c1 ...) (c0.lo.z, c0.hi.z,
// c1.lo.z, c1.hi.z) (ref0, ref1, -, -)
template <>
__device__ __forceinline__ void node_pair<XTGPU_NODES_FP32>(const void *nodes, int32_t i, const RayPre &r, float tmin,
                                                            float tmax, Pair &P)
{
    const float4 *p = (const float4 *)nodes + 4 * (size_t)i;
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    P.h0 = slab_t(fmaf(a.x, r.inv.x, -r.oinv.x), fmaf(a.y, r.inv.x, -r.oinv.x), fmaf(a.z, r.inv.y, -r.oinv.y),
                  fmaf(a.w, r.inv.y, -r.oinv.y), fmaf(c.x, r.inv.z, -r.oinv.z), fmaf(c.y, r.inv.z, -r.oinv.z), tmin,
                  tmax, XTG_TFAR_SCALE, P.t0);
    P.h1 = slab_t(fmaf(b.x, r.inv.x, -r.oinv.x), fmaf(b.y, r.inv.x, -r.oinv.x), fmaf(b.z, r.inv.y, -r.oinv.y),
                  fmaf(b.w, r.inv.y, -r.oinv.y), fmaf(c.z, r.inv.z, -r.oinv.z), fmaf(c.w, r.inv.z, -r.oinv.z), tmin,
                  tmax, XTG_TFAR_SCALE, P.t1);
    P.c0 = __float_as_int(d.x);
    P.c1 = __float_as_int(d.y);
}

// Slightly larger far-distance scale for the quantised test, whose bounds are
// formed in t-space as q * (scale * inv) + (origin * inv - o * inv).
#define XTG_TFAR_SCALE_Q8 1.0000015f

// 32-byte node: origin xyz with a biased power-of-two scale exponent in each
// low byte, 12 child bounds of 8 bits, two child refs.  The slab test runs in
// quantised space: t(q) = q * (s * inv) + (o - ray.o) * inv, one FMA per bound.
template <>
__device__ __forceinline__ void node_pair<XTGPU_NODES_Q8>(const void *nodes, int32_t i, const RayPre &r, float tmin,
                                                          float tmax, Pair &P)
{
    const uint4 *p = (const uint4 *)nodes + 2 * (size_t)i;
    uint4 a = __ldg(p), b = __ldg(p + 1);
    float ax = __uint_as_float((a.x & 0xFFu) << 23) * r.inv.x;
    float ay = __uint_as_float((a.y & 0xFFu) << 23) * r.inv.y;
    float az = __uint_as_float((a.z & 0xFFu) << 23) * r.inv.z;
    float bx = fmaf(__uint_as_float(a.x & ~0xFFu), r.inv.x, -r.oinv.x);
    float by = fmaf(__uint_as_float(a.y & ~0xFFu), r.inv.y, -r.oinv.y);
    float bz = fmaf(__uint_as_float(a.z & ~0xFFu), r.inv.z, -r.oinv.z);
    const uint32_t q0 = a.w, q1 = b.x, q2 = b.y;
#define XTG_Q(w, k) ((float)(((w) >> (8 * (k))) & 0xFFu))
    P.h0 = slab_t(fmaf(XTG_Q(q0, 0), ax, bx), fmaf(XTG_Q(q0, 3), ax, bx), fmaf(XTG_Q(q0, 1), ay, by),
                  fmaf(XTG_Q(q1, 0), ay, by), fmaf(XTG_Q(q0, 2), az, bz), fmaf(XTG_Q(q1, 1), az, bz), tmin, tmax,
                  XTG_TFAR_SCALE_Q8, P.t0);
    P.h1 = slab_t(fmaf(XTG_Q(q1, 2), ax, bx), fmaf(XTG_Q(q2, 1), ax, bx), fmaf(XTG_Q(q1, 3), ay, by),
                  fmaf(XTG_Q(q2, 2), ay, by), fmaf(XTG_Q(q2, 0), az, bz), fmaf(XTG_Q(q2, 3), az, bz), tmin, tmax,
                  XTG_TFAR_SCALE_Q8, P.t1);
#undef XTG_Q
    P.c0 = (int32_t)b.z;
    P.c1 = (int32_t)b.w;
}

// Per-lane view of the scene being traversed.
struct SceneView {
    const void *nodes;
    const float4 *leaf;
    const float4 *planes;
    int32_t root, n_planes;
    uint32_t plane_base;
};

template <int FMT>
__device__ __forceinline__ SceneView scene_view(const DevScene &S)
{
    SceneView v;
    if (FMT == XTGPU_NODES_W8) {
        v.nodes = (const void *)S.nodesW;
        v.leaf = S.leafW;
        v.root = S.rootW;
    } else {
        v.nodes = FMT == XTGPU_NODES_Q8 ? (const void *)S.nodes8 : (const void *)S.nodes32;
        v.leaf = S.leaf_prims;
        v.root = S.root;
    }
    v.planes = S.planes;
    v.n_planes = S.n_planes;
    v.plane_base = (uint32_t)(S.n_tris + S.n_spheres);
    return v;
}

// Primitive i of the leaf array (3 float4: triangle vertices or sphere centre
// and radius, the primitive id in the first w).  All three words are loaded
// before the kind is known, so a triangle waits for one round trip, not two
// (a sphere reads 16 bytes it does not use).
__device__ __forceinline__ void prim_test(const float4 *leaf, uint32_t i, const RayPre &r, float tmin, float &tmax,
                                          uint32_t &prim, float &bu, float &bv)
{
    const float4 *lp = leaf + 3 * (size_t)i;
    const float4 a = __ldg(lp), b = __ldg(lp + 1), c = __ldg(lp + 2);
    uint32_t id = __float_as_uint(a.w);
    if (id & SPHERE_BIT) {
        id &= ~SPHERE_BIT;
        if (hit_sphere(r, make_float3(a.x, a.y, a.z), b.x, tmin, tmax, id, prim)) {
            prim = id;
            bu = bv = 0.f;
        }
    } else {
        float u, v;
        if (hit_triangle(r, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z), make_float3(c.x, c.y, c.z), tmin,
                         tmax, u, v, id, prim)) {
            prim = id;
            bu = u;
            bv = v;
        }
    }
}

// Tests the primitives of leaf `ref`; updates tmax / prim / barycentrics.
__device__ __forceinline__ void leaf_test(const SceneView &V, int32_t ref, const RayPre &r, float tmin, float &tmax,
                                          uint32_t &prim, float &bu, float &bv)
{
    uint32_t first = leaf_first(ref), cnt = leaf_count(ref);
    for (uint32_t k = 0; k < cnt; ++k) prim_test(V.leaf, first + k, r, tmin, tmax, prim, bu, bv);
}

}  // namespace xtg
