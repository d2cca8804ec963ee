// LBVH builder for sm_100a: replaces the reference's only accelerator, the
// per-mesh Octree<Triangle> (src/xtcore/octree.tml:118-198, mesh.cc:70-113),
// with one binary BVH over every triangle and sphere of the scene.
//
//   1. primitive bounds + centroid bounds        (k_prim_bounds)
//   2. 30-bit Morton codes, 10 bits per axis     (k_morton)
//   3. stable LSD radix sort, 4 x 8-bit digits   (k_rs_hist / k_rs_scan / k_rs_scatter)
//   4. Karras 2012 hierarchy                     (k_karras)
//      T. Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees,
//      and k-d Trees", HPG 2012: split search on the common-prefix length of
//      the sorted codes, ties broken by index.
//   5. bottom-up refit with arrival counters     (k_refit)
//   4'-5'. or, with builder 1, PLOC clustering over the same Morton order and
//      a depth-first renumbering of the leaves (k_ploc_*, build_ploc)
//   6. leaf collapse (subtrees of <= leaf_size primitives become one leaf) and
//      FP32 node emission                        (k_emit)
//   7. optional 8-bit quantisation, rounded outward (k_quantise)
//   8. primitives gathered into Morton order     (k_gather)
//
// Steps 2-4 are integer-exact and are checked bit for bit against a CPU
// re-implementation (oracle/lbvh_cpu.c) by the tests.
#include <algorithm>
#include <cmath>

#include "xtgpu_internal.cuh"

namespace xtg {

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;

__device__ __forceinline__ uint32_t f2ord(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ void prim_box(const float4 *tri_v, int n_tris, const float4 *sph, int i, float3 &lo,
                                         float3 &hi)
{
    if (i < n_tris) {
        float4 a = tri_v[3 * i], b = tri_v[3 * i + 1], c = tri_v[3 * i + 2];
        lo = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
        hi = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
    } else {
        float4 s = sph[i - n_tris];
        // rounded outward so the box contains the sphere
        lo = make_float3(__fsub_rd(s.x, s.w), __fsub_rd(s.y, s.w), __fsub_rd(s.z, s.w));
        hi = make_float3(__fadd_ru(s.x, s.w), __fadd_ru(s.y, s.w), __fadd_ru(s.z, s.w));
    }
}

// centroid = (lo + hi) * 0.5 in float, no contraction (the CPU replica matches)
__device__ __forceinline__ float3 centroid(float3 lo, float3 hi)
{
    return make_float3(__fmul_rn(__fadd_rn(lo.x, hi.x), 0.5f), __fmul_rn(__fadd_rn(lo.y, hi.y), 0.5f),
                       __fmul_rn(__fadd_rn(lo.z, hi.z), 0.5f));
}

__global__ void k_prim_bounds(const float4 *tri_v, int n_tris, const float4 *sph, int n, float4 *plo, float4 *phi,
                              uint32_t *cb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float3 c = make_float3(INFINITY, INFINITY, INFINITY), cmx = make_float3(-INFINITY, -INFINITY, -INFINITY);
    if (i < n) {
        float3 lo, hi;
        prim_box(tri_v, n_tris, sph, i, lo, hi);
        plo[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
        phi[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
        c = centroid(lo, hi);
        cmx = c;
    }
    // warp reduce then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        c.x = fminf(c.x, __shfl_xor_sync(0xffffffffu, c.x, o));
        c.y = fminf(c.y, __shfl_xor_sync(0xffffffffu, c.y, o));
        c.z = fminf(c.z, __shfl_xor_sync(0xffffffffu, c.z, o));
        cmx.x = fmaxf(cmx.x, __shfl_xor_sync(0xffffffffu, cmx.x, o));
        cmx.y = fmaxf(cmx.y, __shfl_xor_sync(0xffffffffu, cmx.y, o));
        cmx.z = fmaxf(cmx.z, __shfl_xor_sync(0xffffffffu, cmx.z, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&cb[0], f2ord(c.x));
        atomicMin(&cb[1], f2ord(c.y));
        atomicMin(&cb[2], f2ord(c.z));
        atomicMax(&cb[3], f2ord(cmx.x));
        atomicMax(&cb[4], f2ord(cmx.y));
        atomicMax(&cb[5], f2ord(cmx.z));
    }
}

__device__ __forceinline__ uint32_t expand10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t quant10(float c, float lo, float scale)
{
    float q = __fmul_rn(__fsub_rn(c, lo), scale);
    uint32_t u = (uint32_t)q;   // q >= 0
    return u > 1023u ? 1023u : u;
}

__global__ void k_morton(const float4 *plo, const float4 *phi, int n, const uint32_t *cb, uint32_t *keys,
                         uint32_t *vals)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lox = ord2f(cb[0]), loy = ord2f(cb[1]), loz = ord2f(cb[2]);
    float ex = __fsub_rn(ord2f(cb[3]), lox), ey = __fsub_rn(ord2f(cb[4]), loy), ez = __fsub_rn(ord2f(cb[5]), loz);
    float sx = ex > 0.f ? __fdiv_rn(1024.0f, ex) : 0.f;
    float sy = ey > 0.f ? __fdiv_rn(1024.0f, ey) : 0.f;
    float sz = ez > 0.f ? __fdiv_rn(1024.0f, ez) : 0.f;
    float4 a = plo[i], b = phi[i];
    float3 c = centroid(make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z));
    keys[i] = (expand10(quant10(c.x, lox, sx)) << 2) | (expand10(quant10(c.y, loy, sy)) << 1) |
              expand10(quant10(c.z, loz, sz));
    vals[i] = (uint32_t)i;
}

// --- radix sort -------------------------------------------------------------
__global__ void k_rs_hist(const uint32_t *keys, int n, int shift, uint32_t *hist, int nblocks)
{
    __shared__ uint32_t h[256];
    int t = threadIdx.x;
    h[t] = 0;
    __syncthreads();
    int base = blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int r = 0; r < RS_ITEMS; ++r) {
        int idx = base + r * RS_THREADS + t;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[t * nblocks + blockIdx.x] = h[t];
}

// exclusive scan of `total` counters, one block of 1024 threads
__global__ void k_rs_scan(uint32_t *hist, int total)
{
    __shared__ uint32_t part[1024];
    int t = threadIdx.x;
    int chunk = (total + 1023) / 1024;
    int b = t * chunk, e = min(total, b + chunk);
    uint32_t s = 0;
    for (int i = b; i < e; ++i) s += hist[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        uint32_t v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - s;
    for (int i = b; i < e; ++i) {
        uint32_t v = hist[i];
        hist[i] = run;
        run += v;
    }
}

__global__ void k_rs_scatter(const uint32_t *kin, const uint32_t *vin, uint32_t *kout, uint32_t *vout, int n,
                             int shift, const uint32_t *hist, int nblocks)
{
    __shared__ uint32_t base_off[256];
    __shared__ uint32_t wcount[RS_THREADS / 32][256];
    int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    base_off[t] = hist[t * nblocks + blockIdx.x];
    uint32_t running = 0;   // digit t's count so far in this tile
    uint32_t lt_mask = (1u << lane) - 1u;
    int base = blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ITEMS; ++r) {
        int idx = base + r * RS_THREADS + t;
        bool valid = idx < n;
        uint32_t key = valid ? kin[idx] : 0u;
        uint32_t val = valid ? vin[idx] : 0u;
        uint32_t digit = (key >> shift) & 255u;
#pragma unroll
        for (int w = 0; w < RS_THREADS / 32; ++w) wcount[w][t] = 0;
        __syncthreads();
        uint32_t peers = __match_any_sync(0xffffffffu, valid ? digit : 256u + (uint32_t)lane);
        uint32_t rank = __popc(peers & lt_mask);
        if (valid && rank == 0) wcount[warp][digit] = __popc(peers);
        __syncthreads();
        uint32_t sum = running;
#pragma unroll
        for (int w = 0; w < RS_THREADS / 32; ++w) {
            uint32_t c = wcount[w][t];
            wcount[w][t] = sum;
            sum += c;
        }
        running = sum;
        __syncthreads();
        if (valid) {
            uint32_t pos = base_off[digit] + wcount[warp][digit] + rank;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
    }
}

// --- Karras hierarchy -----------------------------------------------------------
__device__ __forceinline__ int delta(const uint32_t *k, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = k[i], b = k[j];
    return a != b ? __clz(a ^ b) : 32 + __clz((uint32_t)(i ^ j));
}

__global__ void k_karras(const uint32_t *keys, int n, int32_t *left, int32_t *right, int32_t *rlo, int32_t *rhi,
                         int32_t *gam, int32_t *parent_int, int32_t *parent_leaf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int g = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    rlo[i] = lo;
    rhi[i] = hi;
    gam[i] = g;
    if (lo == g) {
        left[i] = ~g;
        parent_leaf[g] = i;
    } else {
        left[i] = g;
        parent_int[g] = i;
    }
    if (hi == g + 1) {
        right[i] = ~(g + 1);
        parent_leaf[g + 1] = i;
    } else {
        right[i] = g + 1;
        parent_int[g + 1] = i;
    }
}

__device__ __forceinline__ void child_box(int32_t ref, const float4 *nlo, const float4 *nhi, const float4 *plo,
                                          const float4 *phi, const uint32_t *order, float4 &lo, float4 &hi)
{
    if (ref >= 0) {
        lo = __ldcg(&nlo[ref]);
        hi = __ldcg(&nhi[ref]);
    } else {
        uint32_t p = order[~ref];
        lo = plo[p];
        hi = phi[p];
    }
}

__global__ void k_refit(int n, const int32_t *left, const int32_t *right, const int32_t *parent_int,
                        const int32_t *parent_leaf, const float4 *plo, const float4 *phi, const uint32_t *order,
                        float4 *nlo, float4 *nhi, int32_t *height, uint32_t *flags)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int node = parent_leaf[k];
    for (int guard = 0; node >= 0; ++guard) {
        if (guard > 256 || node >= n - 1) {   // deeper than any Karras tree of 30-bit codes
            atomicOr(&flags[n - 1], 1u);        // error word just past the arrival counters
            return;
        }
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0u) return;   // the sibling is still on its way
        __threadfence();
        float4 alo, ahi, blo, bhi;
        int32_t l = left[node], r = right[node];
        child_box(l, nlo, nhi, plo, phi, order, alo, ahi);
        child_box(r, nlo, nhi, plo, phi, order, blo, bhi);
        int hl = l >= 0 ? __ldcg(&height[l]) : 0;
        int hr = r >= 0 ? __ldcg(&height[r]) : 0;
        __stcg(&nlo[node], make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.f));
        __stcg(&nhi[node], make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.f));
        __stcg(&height[node], 1 + max(hl, hr));
        node = node == 0 ? -1 : parent_int[node];
    }
}

// Depth-first position of every inner node: the left child follows its parent,
// the right child follows the parent's whole left subtree (g - lo inner nodes).
// Each node climbs to the root summing those offsets.
__global__ void k_dfs_pos(int n, const int32_t *left, const int32_t *rlo, const int32_t *gam,
                          const int32_t *parent_int, int32_t *pos, uint32_t *err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int32_t p = 0, x = i;
    for (int guard = 0; x != 0; ++guard) {
        int32_t par = parent_int[x];
        if (guard > 256 || par < 0 || par >= n - 1) {
            atomicOr(err, 4u);
            return;
        }
        p += left[par] == x ? 1 : 1 + (gam[par] - rlo[par]);
        x = par;
    }
    pos[i] = p;
}

__global__ void k_emit(int n, int leaf_size, const int32_t *left, const int32_t *right, const int32_t *rlo,
                       const int32_t *rhi, const int32_t *gam, const float4 *nlo, const float4 *nhi,
                       const float4 *plo, const float4 *phi, const uint32_t *order, const int32_t *pos, float4 *nodes)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int g = gam[i];
    int32_t l = left[i], r = right[i];
    int nl = g - rlo[i] + 1, nr = rhi[i] - g;
    int32_t refl = nl <= leaf_size ? leaf_ref((uint32_t)rlo[i], (uint32_t)nl) : (pos ? pos[l] : l);
    int32_t refr = nr <= leaf_size ? leaf_ref((uint32_t)(g + 1), (uint32_t)nr) : (pos ? pos[r] : r);
    const int o = pos ? pos[i] : i;
    float4 alo, ahi, blo, bhi;
    child_box(l, nlo, nhi, plo, phi, order, alo, ahi);
    child_box(r, nlo, nhi, plo, phi, order, blo, bhi);
    nodes[4 * o + 0] = make_float4(alo.x, ahi.x, alo.y, ahi.y);
    nodes[4 * o + 1] = make_float4(blo.x, bhi.x, blo.y, bhi.y);
    nodes[4 * o + 2] = make_float4(alo.z, ahi.z, blo.z, bhi.z);
    nodes[4 * o + 3] = make_float4(__int_as_float(refl), __int_as_float(refr), 0.f, 0.f);
}

// Every child reference in range and every leaf range inside the primitive
// array; a violation sets *bad.
__global__ void k_validate(int n, const float4 *nodes, uint32_t *bad)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    float4 r = nodes[4 * i + 3];
    int32_t refs[2] = {__float_as_int(r.x), __float_as_int(r.y)};
    for (int c = 0; c < 2; ++c) {
        int32_t ref = refs[c];
        if (ref >= 0) {
            if (ref >= n - 1 || ref == 0) atomicOr(bad, 1u);
        } else if (ref != EMPTY_REF) {
            uint32_t f = leaf_first(ref), k = leaf_count(ref);
            if (k == 0 || (uint64_t)f + k > (uint64_t)n) atomicOr(bad, 2u);
        }
    }
}

// origin rounded toward -inf with the low 8 mantissa bits cleared
__device__ __forceinline__ uint32_t origin_bits(float v)
{
    uint32_t b = __float_as_uint(v);
    if (v == 0.f) return 0u;
    if (b & 0x80000000u) {
        // negative: round the magnitude up
        uint32_t m = b & 0x7fffffffu;
        m = (m + 0xFFu) & ~0xFFu;
        return m | 0x80000000u;
    }
    return b & ~0xFFu;
}

// smallest biased exponent e (scale 2^(e-127)) with origin + 255*scale >= hi
__device__ __forceinline__ uint32_t pick_exp(float origin, float hi)
{
    float ext = hi - origin;
    uint32_t e = 1;
    if (ext > 0.f) {
        int ex;
        frexpf(ext / 255.0f, &ex);   // ext/255 = m * 2^ex, m in [0.5,1)
        int be = ex + 127;
        e = (uint32_t)max(1, min(254, be - 1));
    }
    // 254 quanta must reach hi
    // one quantum of headroom above hi (the bounds are padded by one quantum)
    while (e < 254 && __fmaf_rn(254.0f, __uint_as_float(e << 23), origin) < hi) ++e;
    return e;
}

__device__ __forceinline__ void quant_axis(float lo, float hi, float o, float sc, uint32_t &qlo, uint32_t &qhi)
{
    if (lo > hi) {   // empty child: inverted box, never hit
        qlo = 255;
        qhi = 0;
        return;
    }
    float a = floorf(__fdiv_rd(__fsub_rd(lo, o), sc));
    float b = ceilf(__fdiv_ru(__fsub_ru(hi, o), sc));
    int ql = (int)fmaxf(0.f, fminf(255.f, a));
    int qh = (int)fmaxf(0.f, fminf(255.f, b));
    while (ql > 0 && __fmaf_rn((float)ql, sc, o) > lo) --ql;
    while (qh < 255 && __fmaf_rn((float)qh, sc, o) < hi) ++qh;
    // one quantum of padding on each side: the traversal evaluates the bounds
    // in t-space with different rounding than this dequantisation
    qlo = (uint32_t)max(0, ql - 1);
    qhi = (uint32_t)min(255, qh + 1);
}

__global__ void k_quantise(int nnodes, const float4 *nodes, uint4 *q)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnodes) return;
    float4 n0 = nodes[4 * i], n1 = nodes[4 * i + 1], n2 = nodes[4 * i + 2], n3 = nodes[4 * i + 3];
    // child a: x [n0.x,n0.y] y [n0.z,n0.w] z [n2.x,n2.y]; child b: x [n1.x,n1.y] y [n1.z,n1.w] z [n2.z,n2.w]
    float lo[3] = {fminf(n0.x, n1.x), fminf(n0.z, n1.z), fminf(n2.x, n2.z)};
    float hi[3] = {fmaxf(n0.y, n1.y), fmaxf(n0.w, n1.w), fmaxf(n2.y, n2.w)};
    float clo[2][3] = {{n0.x, n0.z, n2.x}, {n1.x, n1.z, n2.z}};
    float chi[2][3] = {{n0.y, n0.w, n2.y}, {n1.y, n1.w, n2.w}};
    uint32_t ob[3], ex[3];
    float o[3], sc[3];
    for (int a = 0; a < 3; ++a) {
        float l = lo[a] <= hi[a] ? lo[a] : 0.f;
        float h = lo[a] <= hi[a] ? hi[a] : 0.f;
        ob[a] = origin_bits(l);
        o[a] = __uint_as_float(ob[a]);
        ex[a] = pick_exp(o[a], h);
        sc[a] = __uint_as_float(ex[a] << 23);
    }
    uint32_t qb[12];
    for (int c = 0; c < 2; ++c)
        for (int a = 0; a < 3; ++a) quant_axis(clo[c][a], chi[c][a], o[a], sc[a], qb[c * 6 + a], qb[c * 6 + 3 + a]);
    uint4 w0, w1;
    w0.x = ob[0] | ex[0];
    w0.y = ob[1] | ex[1];
    w0.z = ob[2] | ex[2];
    w0.w = qb[0] | (qb[1] << 8) | (qb[2] << 16) | (qb[3] << 24);
    w1.x = qb[4] | (qb[5] << 8) | (qb[6] << 16) | (qb[7] << 24);
    w1.y = qb[8] | (qb[9] << 8) | (qb[10] << 16) | (qb[11] << 24);
    w1.z = __float_as_uint(n3.x);
    w1.w = __float_as_uint(n3.y);
    q[2 * i] = w0;
    q[2 * i + 1] = w1;
}

__global__ void k_gather(int n, int n_tris, const uint32_t *order, const float4 *tri_v, const float4 *sph,
                         float4 *out)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t p = order[k];
    if ((int)p < n_tris) {
        float4 a = tri_v[3 * p], b = tri_v[3 * p + 1], c = tri_v[3 * p + 2];
        out[3 * k] = make_float4(a.x, a.y, a.z, __uint_as_float(p));
        out[3 * k + 1] = make_float4(b.x, b.y, b.z, 0.f);
        out[3 * k + 2] = make_float4(c.x, c.y, c.z, 0.f);
    } else {
        float4 s = sph[p - n_tris];
        out[3 * k] = make_float4(s.x, s.y, s.z, __uint_as_float(p | SPHERE_BIT));
        out[3 * k + 1] = make_float4(s.w, 0.f, 0.f, 0.f);
        out[3 * k + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// --- PLOC hierarchy ---------------------------------------------------------
// D. Meister and J. Bittner, "Parallel Locally-Ordered Clustering for Bounding
// Volume Hierarchy Construction", IEEE TVCG 24(3), 2018.  The clusters start as
// the leaves in Morton order.  Each iteration every cluster finds, among the
// clusters within PLOC_R positions, the one whose merged box has the smallest
// surface area (ties by ploc_tie); mutual nearest neighbours merge into a new
// internal node at the lower position; the survivors are compacted in order.
// The least pair under (area, ploc_tie) is mutual, so every iteration merges.  Internal nodes are numbered
// from n-2 down, in iteration order and by position within one, so the last
// merge (the root) is node 0 and children have larger indices than parents.
constexpr int PLOC_R = 16;
constexpr int PLOC_T = 256;   // clusters per block of the neighbour search

__device__ __forceinline__ float half_area(float4 alo, float4 ahi, float4 blo, float4 bhi)
{
    // rounded operation by operation, so a CPU replica reproduces every choice
    const float dx = __fsub_rn(fmaxf(ahi.x, bhi.x), fminf(alo.x, blo.x));
    const float dy = __fsub_rn(fmaxf(ahi.y, bhi.y), fminf(alo.y, blo.y));
    const float dz = __fsub_rn(fmaxf(ahi.z, bhi.z), fminf(alo.z, blo.z));
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

// Tie order of the pair {i, j}, the same from both ends: nearer positions
// first, then pairs starting at an even position, then the lower position.
// Equal boxes (duplicated primitives) thus merge (0,1) (2,3) ... at once, and
// as the order over pairs is total, the least pair is always mutual.
__device__ __forceinline__ uint64_t ploc_tie(int i, int j)
{
    const uint32_t lo = (uint32_t)min(i, j), d = (uint32_t)abs(i - j);
    return ((uint64_t)d << 33) | ((uint64_t)(lo & 1u) << 32) | lo;
}

__global__ void k_ploc_init(int n, const float4 *plo, const float4 *phi, const uint32_t *order, float4 *clo,
                            float4 *chi, int32_t *cid)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = order[i];
    clo[i] = plo[p];
    chi[i] = phi[p];
    cid[i] = ~i;
}

__global__ void __launch_bounds__(PLOC_T) k_ploc_nn(int m, const float4 *clo, const float4 *chi, int32_t *nn)
{
    __shared__ float4 slo[PLOC_T + 2 * PLOC_R], shi[PLOC_T + 2 * PLOC_R];
    const int base = blockIdx.x * PLOC_T;
    for (int t = threadIdx.x; t < PLOC_T + 2 * PLOC_R; t += blockDim.x) {
        const int g = base - PLOC_R + t;
        if (g >= 0 && g < m) {
            slo[t] = clo[g];
            shi[t] = chi[g];
        }
    }
    __syncthreads();
    const int i = base + threadIdx.x;
    if (i >= m) return;
    const float4 alo = slo[threadIdx.x + PLOC_R], ahi = shi[threadIdx.x + PLOC_R];
    float best = INFINITY;
    uint64_t bkey = ~0ull;
    int bj = -1;
    for (int o = -PLOC_R; o <= PLOC_R; ++o) {
        const int j = i + o;
        if (o == 0 || j < 0 || j >= m) continue;
        const float a = half_area(alo, ahi, slo[threadIdx.x + PLOC_R + o], shi[threadIdx.x + PLOC_R + o]);
        const uint64_t key = ploc_tie(i, j);
        if (a < best || (a == best && key < bkey)) {
            best = a;
            bkey = key;
            bj = j;
        }
    }
    nn[i] = bj;
}

// per cluster: merges (the lower of a mutual pair) in the low word, survives
// (not absorbed by a lower partner) in the high word
__global__ void k_ploc_flags(int m, const int32_t *nn, unsigned long long *f)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    f[i] = (unsigned long long)(mutual && i < j) | ((unsigned long long)!(mutual && i > j) << 32);
}

__global__ void k_ploc_write(int m, int base, const int32_t *nn, const unsigned long long *ex, const float4 *clo,
                             const float4 *chi, const int32_t *cid, float4 *olo, float4 *ohi, int32_t *oid,
                             int32_t *left, int32_t *right, float4 *nlo, float4 *nhi, int32_t *cnt, int32_t *height,
                             int32_t *pint, int32_t *pleaf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    if (mutual && i > j) return;   // absorbed by its lower partner
    const unsigned long long e = ex[i];
    const int pos = (int)(e >> 32);
    if (!mutual) {
        olo[pos] = clo[i];
        ohi[pos] = chi[i];
        oid[pos] = cid[i];
        return;
    }
    const int k = base - 1 - (int)(e & 0xffffffffull);
    const int32_t a = cid[i], b = cid[j];
    const float4 alo = clo[i], ahi = chi[i], blo = clo[j], bhi = chi[j];
    const float4 lo = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.f);
    const float4 hi = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.f);
    left[k] = a;
    right[k] = b;
    nlo[k] = lo;
    nhi[k] = hi;
    cnt[k] = (a < 0 ? 1 : cnt[a]) + (b < 0 ? 1 : cnt[b]);
    height[k] = 1 + max(a < 0 ? 0 : height[a], b < 0 ? 0 : height[b]);
    if (a < 0) pleaf[~a] = k;
    else pint[a] = k;
    if (b < 0) pleaf[~b] = k;
    else pint[b] = k;
    olo[pos] = lo;
    ohi[pos] = hi;
    oid[pos] = k;
}

// Exclusive scan of 64-bit counters: tiles of 1024 per block, then the tile
// sums (one block), then the offsets added.
constexpr int SCAN_T = 1024;
__device__ __forceinline__ unsigned long long block_scan_ex(unsigned long long v, unsigned long long *sw,
                                                            unsigned long long &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sw[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned long long t = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        sw[lane] = t;   // inclusive warp sums
    }
    __syncthreads();
    total = sw[(blockDim.x >> 5) - 1];
    const unsigned long long before = w ? sw[w - 1] : 0ull;
    return before + x - v;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(int m, const unsigned long long *in, unsigned long long *out,
                                                       unsigned long long *sums)
{
    __shared__ unsigned long long sw[32];
    const int i = blockIdx.x * SCAN_T + threadIdx.x;
    const unsigned long long v = i < m ? in[i] : 0ull;
    unsigned long long total;
    const unsigned long long e = block_scan_ex(v, sw, total);
    if (i < m) out[i] = e;
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// one block: exclusive scan of the tile sums in place, the grand total after them
__global__ void __launch_bounds__(SCAN_T) k_scan_sums(int ntiles, unsigned long long *sums)
{
    __shared__ unsigned long long sw[32];
    unsigned long long carry = 0;
    for (int base = 0; base < ntiles; base += SCAN_T) {
        const int i = base + threadIdx.x;
        const unsigned long long v = i < ntiles ? sums[i] : 0ull;
        unsigned long long total;
        const unsigned long long e = block_scan_ex(v, sw, total);
        __syncthreads();
        if (i < ntiles) sums[i] = carry + e;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[ntiles] = carry;
}

__global__ void k_scan_add(int m, unsigned long long *out, const unsigned long long *sums)
{
    const int i = blockIdx.x * SCAN_T + threadIdx.x;
    if (i < m) out[i] += sums[blockIdx.x];
}

// Leaf offset of a node in the depth-first order of the finished tree: the
// leaves of every left sibling on its way to the root.
__device__ __forceinline__ int ploc_offset(int32_t child, int32_t node, const int32_t *left, const int32_t *right,
                                           const int32_t *cnt, const int32_t *pint, uint32_t *err)
{
    int off = 0;
    for (int guard = 0;; ++guard) {
        if (guard > 4096 || node < 0) {
            atomicOr(err, 8u);
            return 0;
        }
        if (right[node] == child) {
            const int32_t l = left[node];
            off += l < 0 ? 1 : cnt[l];
        }
        if (node == 0) return off;
        child = node;
        node = pint[node];
    }
}

// Inner node ranges of the depth-first leaf order (lo, hi, split as the
// Karras arrays give them) and every leaf's new position.
__global__ void k_ploc_ranges(int n, const int32_t *left, const int32_t *right, const int32_t *cnt,
                              const int32_t *pint, const int32_t *pleaf, int32_t *rlo, int32_t *rhi, int32_t *gam,
                              int32_t *newpos, uint32_t *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n - 1) {
        const int off = i == 0 ? 0 : ploc_offset(i, pint[i], left, right, cnt, pint, err);
        const int32_t l = left[i];
        rlo[i] = off;
        rhi[i] = off + cnt[i] - 1;
        gam[i] = off + (l < 0 ? 1 : cnt[l]) - 1;
    }
    if (i < n) newpos[i] = ploc_offset(~i, pleaf[i], left, right, cnt, pint, err);
}

// Leaf references, Morton keys, primitive order and leaf parents in the new
// leaf order.
__global__ void k_ploc_relabel(int n, int32_t *left, int32_t *right, const int32_t *newpos, const uint32_t *keys,
                               const uint32_t *order, const int32_t *pleaf, uint32_t *keys2, uint32_t *order2,
                               int32_t *pleaf2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n - 1) {
        if (left[i] < 0) left[i] = ~newpos[~left[i]];
        if (right[i] < 0) right[i] = ~newpos[~right[i]];
    }
    if (i < n) {
        const int q = newpos[i];
        keys2[q] = keys[i];
        order2[q] = order[i];
        pleaf2[q] = pleaf[i];
    }
}

struct Tmp {
    cudaStream_t s;
    void *ptrs[64];
    int n = 0;
    ~Tmp()
    {
        for (int i = 0; i < n; ++i) cudaFreeAsync(ptrs[i], s);
    }
    template <class T>
    cudaError_t get(T **p, size_t count)
    {
        cudaError_t e = cudaMallocAsync((void **)p, std::max<size_t>(count, 1) * sizeof(T), s);
        if (e == cudaSuccess) ptrs[n++] = *p;
        return e;
    }
};

inline int blocks(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// PLOC over the Morton order (see k_ploc_nn): fills left/right, the inner
// boxes, heights and parents, then renumbers the leaves in depth-first order
// (keys, order and leaf parents permuted) and gives every inner node its leaf
// range and split as k_karras does, so the rest of the build is shared.
static xtgpu_status build_ploc(int n, cudaStream_t s, Tmp &tmp, const float4 *plo, const float4 *phi,
                               uint32_t *keys, uint32_t *vals, uint32_t *k2, uint32_t *v2, int32_t *left,
                               int32_t *right, int32_t *rlo, int32_t *rhi, int32_t *gam, int32_t *pint, int32_t *pleaf,
                               int32_t *height, float4 *nlo, float4 *nhi, uint32_t *err)
{
    const int ni = n - 1;
    float4 *clo[2], *chi[2];
    int32_t *cid[2], *nn, *cnt, *newpos, *pleaf2;
    unsigned long long *flg, *ex, *sums;
    for (int k = 0; k < 2; ++k) {
        XTG_CUDA(tmp.get(&clo[k], n));
        XTG_CUDA(tmp.get(&chi[k], n));
        XTG_CUDA(tmp.get(&cid[k], n));
    }
    XTG_CUDA(tmp.get(&nn, n));
    XTG_CUDA(tmp.get(&cnt, ni));
    XTG_CUDA(tmp.get(&newpos, n));
    XTG_CUDA(tmp.get(&pleaf2, n));
    XTG_CUDA(tmp.get(&flg, n));
    XTG_CUDA(tmp.get(&ex, n));
    XTG_CUDA(tmp.get(&sums, blocks(n, SCAN_T) + 1));
    unsigned long long *total_h = nullptr;
    XTG_CUDA(cudaMallocHost((void **)&total_h, sizeof(unsigned long long)));
    k_ploc_init<<<blocks(n, 256), 256, 0, s>>>(n, plo, phi, vals, clo[0], chi[0], cid[0]);
    int m = n, base = ni, cur = 0;
    xtgpu_status st = XTGPU_OK;
    for (int it = 0; m > 1; ++it) {
        if (it > 100000) {   // every iteration merges; a bound all the same
            set_error("xtgpu_bvh_build: PLOC did not finish");
            st = XTGPU_ERR_CUDA;
            break;
        }
        const int nt = blocks(m, SCAN_T);
        k_ploc_nn<<<blocks(m, PLOC_T), PLOC_T, 0, s>>>(m, clo[cur], chi[cur], nn);
        k_ploc_flags<<<blocks(m, 256), 256, 0, s>>>(m, nn, flg);
        k_scan_tiles<<<nt, SCAN_T, 0, s>>>(m, flg, ex, sums);
        k_scan_sums<<<1, SCAN_T, 0, s>>>(nt, sums);
        k_scan_add<<<nt, SCAN_T, 0, s>>>(m, ex, sums);
        cudaError_t e = cudaMemcpyAsync(total_h, sums + nt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "PLOC", __FILE__, __LINE__);
            break;
        }
        const int merges = (int)(*total_h & 0xffffffffull), next = (int)(*total_h >> 32);
        if (merges <= 0 || merges > base || next != m - merges) {
            set_error("xtgpu_bvh_build: PLOC made no progress (non-finite primitive bounds?)");
            st = XTGPU_ERR_CUDA;
            break;
        }
        k_ploc_write<<<blocks(m, 256), 256, 0, s>>>(m, base, nn, ex, clo[cur], chi[cur], cid[cur], clo[1 - cur],
                                                    chi[1 - cur], cid[1 - cur], left, right, nlo, nhi, cnt, height,
                                                    pint, pleaf);
        cur = 1 - cur;
        base -= merges;
        m = next;
    }
    cudaFreeHost(total_h);
    if (st != XTGPU_OK) return st;
    if (base != 0) {
        set_error("xtgpu_bvh_build: PLOC left inner nodes unnumbered");
        return XTGPU_ERR_CUDA;
    }
    k_ploc_ranges<<<blocks(n, 256), 256, 0, s>>>(n, left, right, cnt, pint, pleaf, rlo, rhi, gam, newpos, err);
    k_ploc_relabel<<<blocks(n, 256), 256, 0, s>>>(n, left, right, newpos, keys, vals, pleaf, k2, v2, pleaf2);
    XTG_CUDA(cudaMemcpyAsync(keys, k2, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(vals, v2, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(pleaf, pleaf2, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
    return XTGPU_OK;
}

xtgpu_status build_bvh(xtgpu_scene *sc, int node_format, int leaf_size, int layout, cudaStream_t s, int builder)
{
    DevScene &S = sc->dev;
    const int n = S.n_tris + S.n_spheres;
    if ((int64_t)S.n_tris + S.n_spheres >= (1ll << (31 - LEAF_BITS))) {
        set_error("xtgpu_bvh_build: too many primitives");
        return XTGPU_ERR_INVALID;
    }
    leaf_size = std::max(1, std::min(MAX_LEAF, leaf_size));
    sc->n_prims = n;

    // Morton order, keys and topology are the same for both node formats: build
    // them once and keep them.
    bool need_topology = !(sc->built32 || sc->built8) || sc->leaf_size != leaf_size || sc->layout != layout ||
                         sc->builder != builder;
    if (need_topology) {
        sc->built32 = sc->built8 = sc->builtW = false;
        dfree(sc->nodes32);
        dfree(sc->nodes8);
        dfree(sc->nodesW);
        dfree(sc->leafW);
        dfree(sc->leaf_prims);
        dfree(sc->morton);
        dfree(sc->order);
        dfree(sc->left);
        dfree(sc->right);
        sc->leaf_size = leaf_size;
        sc->layout = layout;
        sc->builder = builder;
        if (n == 0) {
            S.root = EMPTY_REF;
            sc->depth = 0;
        } else {
            Tmp tmp{s};
            float4 *plo, *phi;
            uint32_t *cb, *k2, *v2, *hist;
            XTG_CUDA(tmp.get(&plo, n));
            XTG_CUDA(tmp.get(&phi, n));
            XTG_CUDA(tmp.get(&cb, 6));
            XTG_TRY(dalloc(sc->morton, sizeof(uint32_t) * (size_t)n, s));
            XTG_TRY(dalloc(sc->order, sizeof(uint32_t) * (size_t)n, s));
            XTG_TRY(dalloc(sc->leaf_prims, sizeof(float4) * 3 * (size_t)n, s));
            uint32_t *keys = (uint32_t *)sc->morton.p, *vals = (uint32_t *)sc->order.p;
            XTG_CUDA(tmp.get(&k2, n));
            XTG_CUDA(tmp.get(&v2, n));
            uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
            XTG_CUDA(cudaMemcpyAsync(cb, init, sizeof(init), cudaMemcpyHostToDevice, s));
            k_prim_bounds<<<blocks(n, 256), 256, 0, s>>>(S.tri_v, S.n_tris, S.spheres, n, plo, phi, cb);
            k_morton<<<blocks(n, 256), 256, 0, s>>>(plo, phi, n, cb, keys, vals);
            int nb = blocks(n, RS_TILE);
            XTG_CUDA(tmp.get(&hist, (size_t)nb * 256));
            uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
            for (int shift = 0; shift < 32; shift += 8) {
                k_rs_hist<<<nb, RS_THREADS, 0, s>>>(ka, n, shift, hist, nb);
                k_rs_scan<<<1, 1024, 0, s>>>(hist, nb * 256);
                k_rs_scatter<<<nb, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, hist, nb);
                std::swap(ka, kb);
                std::swap(va, vb);
            }
            // 4 passes: the sorted data is back in keys/vals
            XTG_TRY(dalloc(sc->left, sizeof(int32_t) * (size_t)std::max(1, n - 1), s));
            XTG_TRY(dalloc(sc->right, sizeof(int32_t) * (size_t)std::max(1, n - 1), s));
            int32_t *left = (int32_t *)sc->left.p, *right = (int32_t *)sc->right.p;
            if (builder != 1 || n < 2)
                k_gather<<<blocks(n, 256), 256, 0, s>>>(n, S.n_tris, vals, S.tri_v, S.spheres,
                                                        (float4 *)sc->leaf_prims.p);
            S.leaf_prims = (const float4 *)sc->leaf_prims.p;
            if (n == 1) {
                S.root = leaf_ref(0, 1u);
                sc->depth = 0;
                // a single dummy node keeps the node pointers valid
                XTG_TRY(dalloc(sc->nodes32, sizeof(float4) * 4, s));
                XTG_CUDA(cudaMemsetAsync(sc->nodes32.p, 0, sizeof(float4) * 4, s));
            } else {
                int ni = n - 1;
                int32_t *rlo, *rhi, *gam, *pint, *pleaf, *height;
                uint32_t *flags;
                float4 *nlo, *nhi;
                XTG_CUDA(tmp.get(&rlo, ni));
                XTG_CUDA(tmp.get(&rhi, ni));
                XTG_CUDA(tmp.get(&gam, ni));
                XTG_CUDA(tmp.get(&pint, ni));
                XTG_CUDA(tmp.get(&pleaf, n));
                XTG_CUDA(tmp.get(&height, ni));
                XTG_CUDA(tmp.get(&flags, ni + 2));
                XTG_CUDA(tmp.get(&nlo, ni));
                XTG_CUDA(tmp.get(&nhi, ni));
                XTG_CUDA(cudaMemsetAsync(flags, 0, sizeof(uint32_t) * (ni + 2), s));
                XTG_CUDA(cudaMemsetAsync(pint, 0xff, sizeof(int32_t) * ni, s));
                if (builder == 1) {
                    XTG_TRY(build_ploc(n, s, tmp, plo, phi, keys, vals, k2, v2, left, right, rlo, rhi, gam, pint,
                                       pleaf, height, nlo, nhi, flags + ni + 1));
                    // primitives in the new leaf order
                    k_gather<<<blocks(n, 256), 256, 0, s>>>(n, S.n_tris, vals, S.tri_v, S.spheres,
                                                            (float4 *)sc->leaf_prims.p);
                } else {
                    k_karras<<<blocks(ni, 256), 256, 0, s>>>(keys, n, left, right, rlo, rhi, gam, pint, pleaf);
                    k_refit<<<blocks(n, 256), 256, 0, s>>>(n, left, right, pint, pleaf, plo, phi, vals, nlo, nhi,
                                                           height, flags);
                }
                XTG_TRY(dalloc(sc->nodes32, sizeof(float4) * 4 * (size_t)ni, s));
                int32_t *pos = nullptr;
                if (layout == 1) {
                    XTG_CUDA(tmp.get(&pos, ni));
                    k_dfs_pos<<<blocks(ni, 256), 256, 0, s>>>(n, left, rlo, gam, pint, pos, flags + ni + 1);
                }
                k_emit<<<blocks(ni, 256), 256, 0, s>>>(n, leaf_size, left, right, rlo, rhi, gam, nlo, nhi, plo, phi,
                                                       vals, pos, (float4 *)sc->nodes32.p);
                k_validate<<<blocks(ni, 256), 256, 0, s>>>(n, (const float4 *)sc->nodes32.p, flags + ni + 1);
                int32_t h = 0;
                uint32_t errs[2] = {0, 0};
                XTG_CUDA(cudaMemcpyAsync(&h, height, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
                XTG_CUDA(cudaMemcpyAsync(errs, flags + ni, sizeof(errs), cudaMemcpyDeviceToHost, s));
                XTG_CUDA(cudaStreamSynchronize(s));
                if (errs[0] || errs[1]) {
                    sc->built32 = sc->built8 = false;
                    set_error("xtgpu_bvh_build: hierarchy check failed");
                    return XTGPU_ERR_CUDA;
                }
                sc->depth = h;
                // a scene no larger than one leaf is traversed as that leaf
                S.root = n <= leaf_size ? leaf_ref(0, (uint32_t)n) : 0;
            }
            XTG_CUDA(cudaGetLastError());
        }
        S.nodes32 = (const float4 *)sc->nodes32.p;
        sc->built32 = true;
    }
    if (node_format == XTGPU_NODES_Q8 && !sc->built8) {
        int nnodes = (int)(sc->nodes32.bytes / (sizeof(float4) * 4));
        if (nnodes > 0) {
            XTG_TRY(dalloc(sc->nodes8, sizeof(uint4) * 2 * (size_t)nnodes, s));
            k_quantise<<<blocks(nnodes, 256), 256, 0, s>>>(nnodes, (const float4 *)sc->nodes32.p, (uint4 *)sc->nodes8.p);
            XTG_CUDA(cudaGetLastError());
        }
        S.nodes8 = (const uint4 *)sc->nodes8.p;
        sc->built8 = true;
    }
    if (sc->depth > STACK_MAX - 2) {   // the 64-entry stack variant must hold the tree
        set_error("xtgpu_bvh_build: BVH depth exceeds the traversal stack");
        return XTGPU_ERR_LIMIT;
    }
    // the 8-wide nodes again when the collapse asked for differs from the built one
    const xtgpu_tuning &TW = scene_tuning(sc);
    if (node_format == XTGPU_NODES_W8 &&
        (!sc->builtW || sc->wide_collapse != TW.wide_collapse || sc->wide_prim_cost != TW.wide_prim_cost))
        XTG_TRY(build_wide(sc, s));
    sc->last_format = node_format;
    XTG_CUDA(cudaStreamSynchronize(s));
    return XTGPU_OK;
}

}  // namespace xtg
