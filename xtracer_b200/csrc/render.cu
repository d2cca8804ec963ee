// Wavefront kernels and the wave runner shared by xtgpu_render (one job) and
// the render service (many jobs merged per wave).
//
// Per-sample semantics restated from the reference (paths relative to the
// XTracer source tree):
//   camera      Perspective::get_primary_ray, camera/perspective.cc:38-98, in
//               FP64 with every operation rounded as the reference rounds it
//   stencil     integrator/stencil/integrator.cc:13-33
//   depth       integrator/depth/integrator.cc:15-54
//   ao          integrator/ao/integrator.cc:14-52 (maximum distance a parameter)
//   pathtracer  integrator/pathtracer/integrator.cc:21-74 and the materials'
//               sample_path (material/lambert.cc:30-40, phong.cc:35-55,
//               blinnphong.cc:34-61, emissive.cc:20-27, dielectric.cc:22-31)
//   sampling    lib/nmath/sample.inl:28-107, in FP32
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "render.h"
#include "wide.cuh"

namespace xtg {

// ---------------------------------------------------------------------------
// random stream: SplitMix64 finaliser of (path key + counter)
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t path_key(uint64_t seed, uint64_t path)
{
    return mix64(seed ^ mix64(path + 0x9E3779B97F4A7C15ull));
}
__device__ __forceinline__ float uniform(uint64_t key, uint32_t &ctr)
{
    uint64_t x = mix64(key + (uint64_t)(ctr + 1u) * 0x9E3779B97F4A7C15ull);
    ++ctr;
    return (float)(uint32_t)(x >> 40) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalized(float3 a)
{
    float l = sqrtf(dot3(a, a));
    return l != 0.f ? make_float3(a.x / l, a.y / l, a.z / l) : a;
}
// colour channels are clamped at 0 by every operation (lib/nimg/color.inl:48-61)
__device__ __forceinline__ float c0(float v) { return v < 0.f ? 0.f : v; }
__device__ __forceinline__ float3 cmul(float3 a, float3 b) { return make_float3(c0(a.x * b.x), c0(a.y * b.y), c0(a.z * b.z)); }
__device__ __forceinline__ float3 cmuls(float3 a, float s) { return make_float3(c0(a.x * s), c0(a.y * s), c0(a.z * s)); }

// Perspective::get_primary_ray (camera/perspective.cc:38-98), FP64, no contraction.
// Camera rays in FP64, each operation rounded on its own (no contraction), as
// the reference computes them: Perspective::get_primary_ray (perspective.cc:
// 38-98, with the thin-lens draws of :73-95 when flength > 0), ERP (erp.cc:
// 13-31), ODS (ods.cc:17-40) and Cubemap (cubemap.cc:21-69).  `seed`, `path`
// and `ctr` are the sample's random stream; the lens draws are its first two
// values.
__device__ __forceinline__ double dlen3(const double t[3])
{
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(t[0], t[0]), __dmul_rn(t[1], t[1])), __dmul_rn(t[2], t[2])));
}
__device__ __forceinline__ void dnormalize3(double t[3])
{
    const double len = dlen3(t);
    if (len != 0.0) {
        t[0] = __ddiv_rn(t[0], len);
        t[1] = __ddiv_rn(t[1], len);
        t[2] = __ddiv_rn(t[2], len);
    }
}
// (a*x + b*y + c*z) + w, left to right
__device__ __forceinline__ double dsum4(double a, double x, double b, double y, double c, double z, double w)
{
    return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, x), __dmul_rn(b, y)), __dmul_rn(c, z)), w);
}

__device__ void camera_ray(const DevCamera &c, float x, float y, float w, float h, uint64_t seed, uint64_t path,
                           uint32_t &ctr, float3 &o, float3 &d)
{
    double to[3] = {c.pos[0], c.pos[1], c.pos[2]}, t[3];
    if (c.type == XTGPU_CAM_ERP || c.type == XTGPU_CAM_ODS) {
        double dir[3];
        if (c.type == XTGPU_CAM_ERP) {
            const float phi = (float)__dmul_rn(__dmul_rn((double)__fdiv_rn(x, w), 3.14159265358979323846), 2.0);
            const float theta = (float)__dmul_rn((double)__fdiv_rn(y, h), 3.14159265358979323846);
            const double st = sin((double)theta);
            dir[0] = __dmul_rn(st, cos((double)phi));
            dir[1] = cos((double)theta);
            dir[2] = __dmul_rn(st, sin((double)phi));
        } else {
            const float hh = __fmul_rn(h, .5f);
            const float scale = __fmul_rn(__fmul_rn(c.ipd, .5f), (y < hh) ? -1.f : 1.f);
            if (y > hh) y = __fsub_rn(y, hh);
            const float theta = (float)__dmul_rn((double)__fmul_rn(__fdiv_rn(x, w), 2.f), 3.14159265358979323846);
            const float phi = (float)__dsub_rn(__dmul_rn(3.14159265358979323846, 0.5),
                                               __dmul_rn((double)__fdiv_rn(y, hh), 3.14159265358979323846));
            const double ct = cos((double)theta), st = sin((double)theta), cp = cos((double)phi);
            to[0] = __dadd_rn(__dmul_rn(ct, (double)scale), c.pos[0]);
            to[1] = __dadd_rn(__dmul_rn(0.0, (double)scale), c.pos[1]);
            to[2] = __dadd_rn(__dmul_rn(st, (double)scale), c.pos[2]);
            dir[0] = __dmul_rn(st, cp);
            dir[1] = sin((double)phi);
            dir[2] = __dmul_rn(-ct, cp);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) t[k] = dsum4(c.rot[k][0], dir[0], c.rot[k][1], dir[1], c.rot[k][2], dir[2], c.rot[k][3]);
    } else if (c.type == XTGPU_CAM_CUBEMAP) {
        const unsigned long long face_size = (unsigned long long)h / 6ull;
        const unsigned long long face = face_size ? (unsigned long long)y / face_size : 0ull;
        double cd[3] = {0, 0, 0}, up[3] = {0, 0, 0};
        switch (face) {
        case 0: cd[0] = 1; up[1] = 1; break;
        case 1: cd[0] = -1; up[1] = 1; break;
        case 2: cd[1] = 1; up[2] = -1; break;
        case 3: cd[1] = -1; up[2] = 1; break;
        case 4: cd[2] = 1; up[1] = 1; break;
        case 5: cd[2] = -1; up[1] = 1; break;
        }
        y = __fsub_rn(y, (float)(face * face_size));
        double v[3] = {__dsub_rn(__ddiv_rn(__dmul_rn(2.0, (double)x), (double)w), 1.0),
                       __dsub_rn(__ddiv_rn(__dmul_rn(2.0, (double)y), (double)face_size), 1.0), 1.0};
        dnormalize3(v);
        double rx[3] = {__dsub_rn(__dmul_rn(up[1], cd[2]), __dmul_rn(up[2], cd[1])),
                        __dsub_rn(__dmul_rn(up[2], cd[0]), __dmul_rn(up[0], cd[2])),
                        __dsub_rn(__dmul_rn(up[0], cd[1]), __dmul_rn(up[1], cd[0]))};
        dnormalize3(rx);
        double ry[3] = {__dsub_rn(__dmul_rn(rx[1], cd[2]), __dmul_rn(rx[2], cd[1])),
                        __dsub_rn(__dmul_rn(rx[2], cd[0]), __dmul_rn(rx[0], cd[2])),
                        __dsub_rn(__dmul_rn(rx[0], cd[1]), __dmul_rn(rx[1], cd[0]))};
        dnormalize3(ry);
#pragma unroll
        for (int k = 0; k < 3; ++k) t[k] = dsum4(rx[k], v[0], ry[k], v[1], cd[k], v[2], 0.0);
    } else {
        const double aspect = __ddiv_rn((double)w, (double)h);
        double dc[3] = {__dsub_rn(__ddiv_rn(__dmul_rn(2.0, (double)x), (double)w), 1.0),
                        __ddiv_rn(__dsub_rn(__ddiv_rn(__dmul_rn(2.0, (double)y), (double)h), 1.0), aspect), c.dz};
        if (c.flength > 0.f) {
            // the lens point: the camera-space direction moved within half the
            // aperture (two prng_c draws, x then y); the ray aims at the point
            // of the focal plane the undisturbed direction meets
            const uint64_t key = path_key(seed, path);
            const double half = (double)__fdiv_rn(c.aperture, 2.f);
            double lo[3] = {dc[0], dc[1], dc[2]};
            const double u0 = (double)uniform(key, ctr), u1 = (double)uniform(key, ctr);
            lo[0] = __dadd_rn(lo[0], __dadd_rn(__dmul_rn(u0, __dsub_rn(half, -half)), -half));
            lo[1] = __dadd_rn(lo[1], __dadd_rn(__dmul_rn(u1, __dsub_rn(half, -half)), -half));
            const double len = dlen3(dc);
            double fd[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double nk = len != 0.0 ? __ddiv_rn(dc[k], len) : dc[k];
                fd[k] = __dsub_rn(__dadd_rn(dc[k], __dmul_rn(nk, (double)c.flength)), lo[k]);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                t[k] = dsum4(c.rx[k], fd[0], c.ry[k], fd[1], c.rz[k], fd[2], 0.0);
                to[k] = __dadd_rn(dsum4(c.rx[k], lo[0], c.ry[k], lo[1], c.rz[k], lo[2], 0.0), c.pos[k]);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) t[k] = dsum4(c.rx[k], dc[0], c.ry[k], dc[1], c.rz[k], dc[2], 0.0);
        }
        dnormalize3(t);
    }
    if (c.type == XTGPU_CAM_CUBEMAP) dnormalize3(t);
    o = make_float3((float)to[0], (float)to[1], (float)to[2]);
    d = make_float3((float)t[0], (float)t[1], (float)t[2]);
}

// Origin moved off the surface along n by a few ulps (Waechter and Binder, "A
// Fast and Robust Method for Avoiding Self-Intersection", Ray Tracing Gems
// 2019); the reference moves it by n * 1e-8, which FP32 cannot resolve.
__device__ __forceinline__ float3 offset_ray(float3 p, float3 n)
{
    const float origin = 1.0f / 32.0f, fscale = 1.0f / 65536.0f, iscale = 256.0f;
    int ix = (int)(iscale * n.x), iy = (int)(iscale * n.y), iz = (int)(iscale * n.z);
    float px = __int_as_float(__float_as_int(p.x) + (p.x < 0.f ? -ix : ix));
    float py = __int_as_float(__float_as_int(p.y) + (p.y < 0.f ? -iy : iy));
    float pz = __int_as_float(__float_as_int(p.z) + (p.z < 0.f ? -iz : iz));
    return make_float3(fabsf(p.x) < origin ? p.x + fscale * n.x : px, fabsf(p.y) < origin ? p.y + fscale * n.y : py,
                       fabsf(p.z) < origin ? p.z + fscale * n.z : pz);
}

// sample::hemisphere (sample.inl:28-59).  cross(n + eps, n) = eps * cross((1,1,1), n).
__device__ float3 s_hemisphere(float3 n, uint64_t key, uint32_t &ctr)
{
    float u = uniform(key, ctr), v = uniform(key, ctr);
    float phi = acosf(sqrtf(u));
    float theta = 6.283185307179586f * v;
    float sp, cp, st, ct;
    sincosf(phi, &sp, &cp);
    sincosf(theta, &st, &ct);
    float3 d = make_float3(ct * sp, cp, st * sp);
    float3 nn = normalized(n);
    float3 xv = normalized(cross3(make_float3(1.f, 1.f, 1.f), nn));
    float3 zv = normalized(cross3(xv, nn));
    return normalized(xv * d.x + nn * d.y + zv * d.z);
}

// sample::diffuse (sample.inl:92-107): rejection on x^4 + y^4 + z^4 < 1; the
// first value drawn is z, as the reference build evaluates the three draws.
__device__ float3 s_diffuse(float3 n, uint64_t key, uint32_t &ctr)
{
    float3 p = make_float3(0.f, 0.f, 0.f);
    for (int it = 0; it < 256; ++it) {
        float c = uniform(key, ctr), b = uniform(key, ctr), a = uniform(key, ctr);
        p = make_float3(2.f * a - 1.f, 2.f * b - 1.f, 2.f * c - 1.f);
        float x2 = p.x * p.x, y2 = p.y * p.y, z2 = p.z * p.z;
        if (x2 * x2 + y2 * y2 + z2 * z2 < 1.0f) break;
    }
    return normalized(p + n);
}

// sample::lobe (sample.inl:61-90) in FP64, step by step: the frame (ivec,
// refl, kvec) as columns, or the identity when 1 - d.n <= 1e-8 (the raw,
// unnormalised vectors, as the reference tests them); then vc * pow(vdotr, e)
// normalised.  Returns false when that product is too small for its length to
// be nonzero in FP64 (vdotr clamped to 0, or pow underflowing, which happens
// with the identity frame, where vc need not lie around the reflection): the
// reference then keeps the unnormalised, zero or subnormal vector as the next
// ray's direction, and that ray meets nothing (every primitive test rejects a
// direction whose dot products are below 1e-8).  `out` is the direction
// rounded to FP32; `twice` normalises it once more first, as
// BlinnPhong::sample_path does (blinnphong.cc:55).  `raw` is the FP64
// vector, which the environment takes in the degenerate case.
__device__ __forceinline__ double ddot3(const double a[3], const double b[3])
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}
__device__ __forceinline__ void dcross3(const double a[3], const double b[3], double r[3])
{
    r[0] = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
    r[1] = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
    r[2] = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
}
__device__ __forceinline__ bool s_lobe(const double n[3], const double d[3], float e, bool twice, uint64_t key,
                                       uint32_t &ctr, float3 &out, double3 &raw)
{
    double i[3] = {d[0], d[1], d[2]}, nn[3] = {n[0], n[1], n[2]};
    dnormalize3(i);
    dnormalize3(nn);
    // Vector3f::reflected (vector.inl:455-460): (2 * dot(i, n) * n) - i
    const double k2 = __dmul_rn(2.0, ddot3(i, nn));
    double refl[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) refl[c] = __dsub_rn(__dmul_rn(k2, nn[c]), i[c]);
    double cx[3] = {1.0, 0.0, 0.0}, cy[3] = {0.0, 1.0, 0.0}, cz[3] = {0.0, 0.0, 1.0};   // Matrix3x3f() = identity
    if (__dsub_rn(1.0, ddot3(d, n)) > 1e-8) {
        dcross3(d, refl, cx);
        dnormalize3(cx);
        cy[0] = refl[0]; cy[1] = refl[1]; cy[2] = refl[2];
        dcross3(refl, cx, cz);
    }
    const double u = (double)uniform(key, ctr), v = (double)uniform(key, ctr);
    const double theta = __dmul_rn(__dmul_rn(2.0, 3.14159265358979323846), u);
    const double phi = acos(pow(v, __ddiv_rn(1.0, __dadd_rn((double)e, 1.0))));
    const double sp = sin(phi), cp = cos(phi), st = sin(theta), ct = cos(theta);
    const double l[3] = {__dmul_rn(ct, sp), cp, __dmul_rn(st, sp)};
    double vc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)   // Vector3f::transformed: the matrix times the column vector
        vc[c] = __dadd_rn(__dadd_rn(__dmul_rn(cx[c], l[0]), __dmul_rn(cy[c], l[1])), __dmul_rn(cz[c], l[2]));
    double vdotr = ddot3(refl, vc);
    if (vdotr < 0.0) vdotr = 0.0;
    const double p = pow(vdotr, (double)e);
    double w[3] = {__dmul_rn(vc[0], p), __dmul_rn(vc[1], p), __dmul_rn(vc[2], p)};
    const double len = dlen3(w);
    raw = make_double3(w[0], w[1], w[2]);
    if (len == 0.0) {
        out = make_float3(0.f, 0.f, 0.f);
        return false;
    }
    w[0] = __ddiv_rn(w[0], len);
    w[1] = __ddiv_rn(w[1], len);
    w[2] = __ddiv_rn(w[2], len);
    if (twice) dnormalize3(w);
    out = make_float3((float)w[0], (float)w[1], (float)w[2]);
    return true;
}


// Hit record normal as the reference forms it: triangles the face normal (or the
// barycentric blend of vertex normals when given, not renormalised), spheres
// (p - c) / r, planes the stored normal.
__device__ __forceinline__ float3 hit_normal(const DevScene &S, uint32_t prim, float3 p, float bu, float bv)
{
    if ((int)prim < S.n_tris) {
        float3 a = f3(S.tri_v[3 * prim]), b = f3(S.tri_v[3 * prim + 1]), c = f3(S.tri_v[3 * prim + 2]);
        float3 fn = normalized(cross3(b - a, c - a));
        if (S.tri_n) {
            float bw = 1.f - bu - bv;
            float3 na = f3(S.tri_n[3 * prim]), nb = f3(S.tri_n[3 * prim + 1]), nc = f3(S.tri_n[3 * prim + 2]);
            float3 pn = na * bw + nb * bu + nc * bv;
            if (dot3(pn, pn) != 0.f) return pn;
        }
        return fn;
    }
    if ((int)prim < S.n_tris + S.n_spheres) {
        float4 s = S.spheres[prim - S.n_tris];
        return make_float3((p.x - s.x) / s.w, (p.y - s.y) / s.w, (p.z - s.z) / s.w);
    }
    return f3(S.planes[prim - S.n_tris - S.n_spheres]);
}

// The hit record's normal in FP64, as the reference forms it from its FP64 hit
// point: triangles the face normal normalised in FP64 from the float vertices
// (Triangle::calc_normal, triangle.cc:142-147), or the barycentric blend of the
// vertex normals when it is not zero; spheres (o + d t - c) / r
// (sphere.cc:52); planes the stored normal.  The FP32 normal's own rounding
// (a few 1e-8 in its length) would decide sample::lobe's 1 - d.n <= 1e-8 test
// for head-on hits differently from the reference.
__device__ void hit_normal_d(const DevScene &S, uint32_t prim, float3 o, float3 d, float t, float bu, float bv,
                             double n[3])
{
    if ((int)prim < S.n_tris) {
        const float4 a = S.tri_v[3 * prim], b = S.tri_v[3 * prim + 1], c = S.tri_v[3 * prim + 2];
        const double e1[3] = {__dsub_rn(b.x, a.x), __dsub_rn(b.y, a.y), __dsub_rn(b.z, a.z)};
        const double e2[3] = {__dsub_rn(c.x, a.x), __dsub_rn(c.y, a.y), __dsub_rn(c.z, a.z)};
        dcross3(e1, e2, n);
        dnormalize3(n);
        if (S.tri_n) {
            const double w0 = 1.0 - (double)bu - (double)bv;
            const float4 na = S.tri_n[3 * prim], nb = S.tri_n[3 * prim + 1], nc = S.tri_n[3 * prim + 2];
            const double pn[3] = {__dadd_rn(__dadd_rn(__dmul_rn(na.x, w0), __dmul_rn(nb.x, bu)), __dmul_rn(nc.x, bv)),
                                  __dadd_rn(__dadd_rn(__dmul_rn(na.y, w0), __dmul_rn(nb.y, bu)), __dmul_rn(nc.y, bv)),
                                  __dadd_rn(__dadd_rn(__dmul_rn(na.z, w0), __dmul_rn(nb.z, bu)), __dmul_rn(nc.z, bv))};
            if (dlen3(pn) != 0.0) {
                n[0] = pn[0]; n[1] = pn[1]; n[2] = pn[2];
            }
        }
        return;
    }
    if ((int)prim < S.n_tris + S.n_spheres) {
        const float4 c = S.spheres[prim - S.n_tris];
        n[0] = __ddiv_rn(__dsub_rn(__dadd_rn(o.x, __dmul_rn(d.x, t)), c.x), c.w);
        n[1] = __ddiv_rn(__dsub_rn(__dadd_rn(o.y, __dmul_rn(d.y, t)), c.y), c.w);
        n[2] = __ddiv_rn(__dsub_rn(__dadd_rn(o.z, __dmul_rn(d.z, t)), c.z), c.w);
        return;
    }
    const float4 pl = S.planes[prim - S.n_tris - S.n_spheres];
    n[0] = pl.x; n[1] = pl.y; n[2] = pl.z;
}

// The specular branch of Phong / BlinnPhong::sample_path (phong.cc:48-52,
// blinnphong.cc:52-56): sample::lobe around the reflection of the incident
// direction, with the hit normal in FP64 and the ray's direction normalised in
// FP64 (the reference's is a normalised double).  Kept out of line: it is the
// only FP64 vector work of the shade kernel.
__device__ __noinline__ bool phong_lobe(const DevScene &S, const xtgpu_hit &h, float3 o, float3 d, float e, bool twice,
                                        uint64_t key, uint32_t &ctr, float3 &out, double3 &raw)
{
    double n[3], dir[3] = {-(double)d.x, -(double)d.y, -(double)d.z};
    hit_normal_d(S, h.prim, o, d, h.t, h.u, h.v, n);
    dnormalize3(dir);
    return s_lobe(n, dir, e, twice, key, ctr, out, raw);
}

// hit_record_t::texcoord as the reference forms it: triangles interpolate
// their corner texcoords (the Triangle constructor's (0,0) (1,0) (0,0) when the
// scene gives none, math/triangle.cc:8-13), spheres asin of the normal over the
// u/v scale (math/sphere.cc:52-53), planes a planar map wrapped into [0,1]
// (math/plane.cc:47-58).  Spheres and planes in FP64 like the reference.
__device__ double2 hit_texcoord_d(const DevScene &S, uint32_t prim, float3 o, float3 d, float t, float bu, float bv)
{
    if ((int)prim < S.n_tris) {
        float2 a = make_float2(0.f, 0.f), b = make_float2(1.f, 0.f), c = make_float2(0.f, 0.f);
        if (S.tri_uv) {
            a = S.tri_uv[3 * prim];
            b = S.tri_uv[3 * prim + 1];
            c = S.tri_uv[3 * prim + 2];
        }
        const double bw = 1.0 - (double)bu - (double)bv;
        return make_double2(a.x * bw + b.x * (double)bu + c.x * (double)bv, a.y * bw + b.y * (double)bu + c.y * (double)bv);
    }
    const float2 sc = S.obj_uvs[S.prim_obj[prim]];
    const double px = (double)o.x + (double)d.x * t, py = (double)o.y + (double)d.y * t,
                 pz = (double)o.z + (double)d.z * t;
    if ((int)prim < S.n_tris + S.n_spheres) {
        const float4 s4 = S.spheres[prim - S.n_tris];
        const double nx = (px - s4.x) / s4.w, ny = (py - s4.y) / s4.w;
        const double PI = 3.14159265358979323846;
        return make_double2(asin(nx / (sc.x != 0.f ? (double)sc.x : 1.0)) / PI + 0.5,
                            asin(ny / (sc.y != 0.f ? (double)sc.y : 1.0)) / PI + 0.5);
    }
    const float4 pl = S.planes[prim - S.n_tris - S.n_spheres];
    const double l = sqrt((double)pl.x * pl.x + (double)pl.y * pl.y + (double)pl.z * pl.z);
    const double nx = pl.x / l, ny = pl.y / l, nz = pl.z / l;
    const double ux = ny, uy = nz, uz = -nx;                                    // uvec
    const double vx = uy * nz - uz * ny, vy = uz * nx - ux * nz, vz = ux * ny - uy * nx;   // cross(uvec, n)
    const double qx = fabs((double)pl.x) * pl.w + px, qy = fabs((double)pl.y) * pl.w + py,
                 qz = fabs((double)pl.z) * pl.w + pz;
    double tu = (ux * qx + uy * qy + uz * qz) * (double)sc.x;
    double tv = (vx * qx + vy * qy + vz * qz) * (double)sc.y;
    if (tu > 1.f) tu -= (float)(int)tu;
    if (tv > 1.f) tv -= (float)(int)tv;
    if (tu < -1.f) tu -= (float)(int)tu;
    if (tv < -1.f) tv -= (float)(int)tv;
    if (tu < 0.f) tu = 1.f + tu;
    if (tv < 0.f) tv = 1.f + tv;
    return make_double2(tu, tv);
}

__device__ __forceinline__ float2 hit_texcoord(const DevScene &S, uint32_t prim, float3 o, float3 d, float t,
                                               float bu, float bv)
{
    const double2 tc = hit_texcoord_d(S, prim, o, d, t, bu, bv);
    return make_float2((float)tc.x, (float)tc.y);
}

// ---------------------------------------------------------------------------
// Samplers (sampler_*.cc) with the reference's arithmetic: every operation
// rounded on its own, colours clamped at 0 after each step (color.inl).

// the x86-64 int conversion of a float (cvttss2si): INT_MIN outside int's
// range and for NaN
__device__ __forceinline__ int f2i_x86(float f)
{
    return (f != f || f >= 2147483648.f || f < -2147483648.f) ? INT_MIN : __float2int_rz(f);
}

// Pixmap::pixel_ro (lib/nimg/pixmap.cc:44-50): coordinates clamped to the
// last column and row
__device__ __forceinline__ float3 texel_at(const DevScene &S, const DevTexture &t, uint64_t x, uint64_t y)
{
    const uint64_t nx = x >= (uint64_t)t.width ? (uint64_t)t.width - 1 : x;
    const uint64_t ny = y >= (uint64_t)t.height ? (uint64_t)t.height - 1 : y;
    const float4 c = __ldg(&S.texels[t.offset + (int64_t)(ny * (uint64_t)t.width + nx)]);
    return make_float3(c.x, c.y, c.z);
}

__device__ __forceinline__ float3 cscale_rn(float3 c, float s)
{
    return make_float3(c0(__fmul_rn(c.x, s)), c0(__fmul_rn(c.y, s)), c0(__fmul_rn(c.z, s)));
}
__device__ __forceinline__ float3 cadd_rn(float3 a, float3 b)
{
    return make_float3(c0(__fadd_rn(a.x, b.x)), c0(__fadd_rn(a.y, b.y)), c0(__fadd_rn(a.z, b.z)));
}

// nimg::sample::nearest (lib/nimg/sample.cc:8-17): wrapped into [0, 1], then
// (size_t)(u * (float)width); NaN converts to 2^63 on x86-64 (the last texel)
__device__ float3 tex_nearest(const DevScene &S, const DevTexture &t, double u, double v)
{
    u = u < 0 ? 0.0 : (u > 1 ? __dsub_rn(u, floor(u)) : u);
    v = v < 0 ? 0.0 : (v > 1 ? __dsub_rn(v, floor(v)) : v);
    const double fx = __dmul_rn(u, (double)(float)t.width), fy = __dmul_rn(v, (double)(float)t.height);
    const uint64_t x = fx == fx ? (uint64_t)fx : (1ull << 63);
    const uint64_t y = fy == fy ? (uint64_t)fy : (1ull << 63);
    return texel_at(S, t, x, y);
}

// ((size_t)i) % n for an int i, as the reference's `int % size_t` computes
// it: a negative i converts to 2^64 + i.  With m = 2^64 mod n (precomputed
// per texture) that is (m + n - (-i mod n)) mod n, all in 32 bits.
__device__ __forceinline__ uint32_t wrap_index(int i, uint32_t n, uint32_t m)
{
    if (i >= 0) return (uint32_t)i % n;
    const uint32_t a = (uint32_t)(-(int64_t)i % (int64_t)n);
    return (uint32_t)(((uint64_t)m + n - a) % n);
}

// nimg::sample::bilinear (lib/nimg/sample.cc:19-52): int texel index modulo
// the size_t size (a negative index wraps through 2^64), weights in float,
// four colours scaled and summed as ColorRGBAf
__device__ float3 tex_bilinear(const DevScene &S, const DevTexture &t, double u, double v)
{
    const uint32_t w = (uint32_t)t.width, h = (uint32_t)t.height;
    const float fu = (float)__dmul_rn(u, (double)w), fv = (float)__dmul_rn(v, (double)h);
    const int u1 = (int)wrap_index(f2i_x86(fu), w, t.wrap_w), v1 = (int)wrap_index(f2i_x86(fv), h, t.wrap_h);
    const int u2 = (int)((uint32_t)(u1 + 1) % w), v2 = (int)((uint32_t)(v1 + 1) % h);
    const float fru = __fsub_rn(fu, floorf(fu)), frv = __fsub_rn(fv, floorf(fv));
    const float iu = __fsub_rn(1.f, fru), iv = __fsub_rn(1.f, frv);
    const float w1 = __fmul_rn(iu, iv), w2 = __fmul_rn(fru, iv), w3 = __fmul_rn(iu, frv), w4 = __fmul_rn(fru, frv);
    float3 c = cadd_rn(cscale_rn(texel_at(S, t, u1, v1), w1), cscale_rn(texel_at(S, t, u2, v1), w2));
    c = cadd_rn(c, cscale_rn(texel_at(S, t, u1, v2), w3));
    return cadd_rn(c, cscale_rn(texel_at(S, t, u2, v2), w4));
}

// Texture2D::sample, sampler_tex.cc:37-45
__device__ __forceinline__ float3 tex_sample(const DevScene &S, int ti, double u, double v)
{
    const DevTexture t = S.textures[ti];
    return t.filtering == XTGPU_FILTER_BILINEAR ? tex_bilinear(S, t, u, v) : tex_nearest(S, t, u, v);
}

// Vector3f::normalized (vector.inl:444-448)
__device__ __forceinline__ void dnormalized(double &x, double &y, double &z)
{
    const double l = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    if (l != 0.0) {
        x = __ddiv_rn(x, l);
        y = __ddiv_rn(y, l);
        z = __ddiv_rn(z, l);
    }
}

// ERP::sample, sampler_erp.cc:13-26 (angles rounded to float)
__device__ float3 erp_sample(const DevScene &S, int ti, double x, double y, double z)
{
    dnormalized(x, y, z);
    const float theta = (float)acos(y);
    const float phi = (float)atan2(x, -z);
    const float u = (float)__dadd_rn(0.5, __ddiv_rn((double)phi, 6.283185307179586232));
    const float v = (float)__ddiv_rn((double)theta, 3.14159265358979323846);
    return tex_sample(S, ti, u, v);
}

// Cubemap::sample, sampler_cubemap.cc:13-36: the face of the largest
// component (CUBEMAP_FACE order: left, right, top, bottom, front, back)
__device__ float3 cube_sample(const DevScene &S, int ti, double x, double y, double z)
{
    dnormalized(x, y, z);
    int face = 2;
    double u = 0.0, v = 0.0;
    const double ax = fabs(x), ay = fabs(y), az = fabs(z);
    auto half = [](double p, double q) { return __dmul_rn(__dadd_rn(__ddiv_rn(p, q), 1.0), 0.5); };
    if (ax >= ay && ax >= az) {
        if (x > 0.0) { face = 1; u = half(z, x); v = __dsub_rn(1.0, half(y, x)); }
        else if (x < 0.0) { face = 0; u = half(z, x); v = half(y, x); }
    } else if (ay >= ax && ay >= az) {
        if (y > 0.0) { face = 2; u = half(x, y); v = __dsub_rn(1.0, half(z, y)); }
        else if (y < 0.0) { face = 3; u = __dsub_rn(1.0, half(x, y)); v = __dsub_rn(1.0, half(z, y)); }
    } else if (az >= ax && az >= ay) {
        if (z > 0.0) { face = 5; u = __dsub_rn(1.0, half(x, z)); v = __dsub_rn(1.0, half(y, z)); }
        else if (z < 0.0) { face = 4; u = __dsub_rn(1.0, half(x, z)); v = half(y, z); }
    }
    // u and v are floats in the reference
    return tex_sample(S, ti + face, (double)(float)u, (double)(float)v);
}

// Gradient::sample, sampler_gradient.cc:11-17, on a direction or texcoord
__device__ float3 gradient_sample(float3 a, float3 b, double x, double y, double z)
{
    dnormalized(x, y, z);
    const float t = (float)__dadd_rn(__dmul_rn(0.5, y), 1.0);
    return cadd_rn(cscale_rn(make_float3(c0(a.x), c0(a.y), c0(a.z)), (float)__dsub_rn(1.0, (double)t)),
                   cscale_rn(make_float3(c0(b.x), c0(b.y), c0(b.z)), t));
}

__device__ float3 sampler_eval(const DevScene &S, const DevSampler &k, double x, double y, double z)
{
    switch (k.kind) {
    case XTGPU_SAMPLER_GRADIENT: return gradient_sample(k.a, k.b, x, y, z);
    case XTGPU_SAMPLER_TEXTURE: return tex_sample(S, k.tex, x, y);
    case XTGPU_SAMPLER_ERP: return erp_sample(S, k.tex, x, y, z);
    case XTGPU_SAMPLER_CUBEMAP: return cube_sample(S, k.tex, x, y, z);
    default: return make_float3(c0(k.a.x), c0(k.a.y), c0(k.a.z));
    }
}

// IMaterial::get_sample (material.cc:65-70) of channel ch (0 diffuse, 1
// specular, 2 emissive) at the hit's texcoord (u, v, 0), which is formed only
// for a textured material
__device__ __forceinline__ float3 mat_color(const DevScene &S, const DevMaterial &M, int ch, const xtgpu_hit &h,
                                            float3 o, float3 d)
{
    if (!M.textured) return ch == 0 ? M.diffuse : (ch == 1 ? M.specular : M.emissive);
    const double2 tc = hit_texcoord_d(S, h.prim, o, d, h.t, h.u, h.v);
    return sampler_eval(S, M.s[ch], tc.x, tc.y, 0.0);
}

// Scene::sample_environment (scene.cc:142-145): black without an environment
__device__ float3 environment_d(const DevScene &S, double x, double y, double z)
{
    switch (S.env_type) {
    case XTGPU_ENV_COLOR: return S.env_a;
    case XTGPU_ENV_GRADIENT: return gradient_sample(S.env_a, S.env_b, x, y, z);
    case XTGPU_ENV_ERP: return erp_sample(S, S.env_tex, x, y, z);
    case XTGPU_ENV_CUBEMAP: return cube_sample(S, S.env_tex, x, y, z);
    default: return make_float3(0.f, 0.f, 0.f);
    }
}
__device__ __forceinline__ float3 environment(const DevScene &S, float3 dir)
{
    return environment_d(S, dir.x, dir.y, dir.z);
}

// Pixel of the k-th pixel slot of a job.  With tiles, slots run through
// square tiles of `tile` pixels (row-major tiles, row-major inside a tile; the
// last band and column may be partial), which keeps the rays of a warp close
// together on screen.  A bijection of [0, rw*rh), so every pixel is visited once.
__device__ __forceinline__ void pixel_of(const DevJob &J, int64_t k, int &x, int &y)
{
    const int T = J.tile;
    if (T <= 1) {
        x = J.x0 + (int)(k % J.rw);
        y = J.y0 + (int)(k / J.rw);
        return;
    }
    const int64_t bandpix = (int64_t)T * J.rw;
    const int64_t band = k / bandpix;
    const int64_t qq = k - band * bandpix;
    const int th = min(T, J.rh - (int)band * T);
    const int64_t c = qq / ((int64_t)T * th);
    const int wc = min(T, J.rw - (int)c * T);
    const int64_t rr = qq - c * T * th;
    y = J.y0 + (int)band * T + (int)(rr / wc);
    x = J.x0 + (int)c * T + (int)(rr % wc);
}

__device__ __forceinline__ int find_job(const DevJob *jobs, int njobs, int64_t i)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].offset <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int warp_append(int32_t *counter, bool pred)
{
    unsigned act = __activemask();
    unsigned m = __ballot_sync(act, pred);
    int lane = threadIdx.x & 31;
    int leader = __ffs(act) - 1;
    int base = 0;
    if (lane == leader && m) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(act, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ const DevScene &scene_of(const DevScene *scenes, const DevJob &j) { return scenes[j.scene]; }

// ---------------------------------------------------------------------------
__global__ void k_camera(const DevJob *__restrict__ jobs, const DevScene *__restrict__ scenes, WaveQueues q)
{
    const int njobs = q.ctl[4];
    const int64_t total = q.ctl[5];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int jn = find_job(jobs, njobs, i);
        const DevJob &J = jobs[jn];
        int64_t p = J.first + (i - J.offset);
        int64_t npix = (int64_t)J.rw * J.rh;
        int64_t s = p / npix, pix = p - s * npix;
        int x, y;
        pixel_of(J, pix, x, y);
        // position of the sample (aa.cc:7-77), each taken spp1 times: the
        // grid's aa^2 (rows in order) or aa jittered ones
        float cx = (float)x + 0.5f, cy = (float)y + 0.5f;
        if (J.dist == XTGPU_SAMPLES_RANDOM) {
            // gen_samples_random (aa.cc:34-48): pixel + (float)prng_c(0, 1) per axis
            const uint64_t jk = path_key(J.seed ^ JITTER_SALT, (uint64_t)(s / J.spp1) * (uint64_t)J.width *
                                                                   (uint64_t)J.height +
                                                               (uint64_t)y * (uint64_t)J.width + (uint64_t)x);
            uint32_t jc = 0;
            const float u = uniform(jk, jc), v = uniform(jk, jc);
            cx = (float)__dadd_rn((double)x, (double)u);
            cy = (float)__dadd_rn((double)y, (double)v);
        } else if (J.aa > 1) {
            const int gi = (int)(s / J.spp1);
            const float sub = __fdiv_rn(1.f, (float)J.aa), off = __fmul_rn(sub, 0.5f);
            cx = (float)__dadd_rn(__dadd_rn((double)x, __dmul_rn((double)(gi % J.aa), (double)sub)), (double)off);
            cy = (float)__dadd_rn(__dadd_rn((double)y, __dmul_rn((double)(gi / J.aa), (double)sub)), (double)off);
        }
        // the sample's random stream, keyed as in k_shade
        const uint64_t path = (uint64_t)s * (uint64_t)J.width * (uint64_t)J.height + (uint64_t)y * (uint64_t)J.width +
                              (uint64_t)x;
        uint32_t ctr = 0;
        float3 o, d;
        camera_ray(scenes[J.scene].cam, cx, cy, (float)J.width, (float)J.height, J.seed, path, ctr, o, d);
        q.org[0][i] = make_float4(o.x, o.y, o.z, 0.f);
        q.dir[0][i] = make_float4(d.x, d.y, d.z, INFINITY);
        q.meta[0][i] = make_uint2((uint32_t)i, (uint32_t)jn);
        // the integrators draw from the stream after the lens draws
        q.P[0][i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(ctr));
        q.I[0][i] = make_float4(1.f, 1.f, 1.f, __int_as_float(J.bounces));
        q.contrib[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// Persistent extend with refill: one node or one leaf per lane per iteration;
// when at least `refill` lanes of the warp have finished their rays they take
// new ones from the queue together (Aila and Laine, "Understanding the
// Efficiency of Ray Traversal on GPUs", HPG 2009: dynamic ray fetch), so long
// rays do not hold a mostly idle warp.
// "pop the next stack entry": a leaf ref of count 0 that no build produces
constexpr int32_t POP_REF = ~(1 << LEAF_BITS);

template <int FMT, bool MULTI>
__global__ void __launch_bounds__(256) k_extend_refill(DevScene S1, const DevScene *__restrict__ scenes,
                                                       const DevJob *__restrict__ jobs, WaveQueues q, int side,
                                                       int refill)
{
    const int n = q.ctl[side];
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(q.rays, (unsigned long long)n);
    const float4 *org = q.org[side], *dir = q.dir[side];
    SceneView V = scene_view<FMT>(S1);
    RayPre r;
    float tmin = 0.f, tmax = 0.f, bu = 0.f, bv = 0.f;
    uint32_t prim = 0xffffffffu, nv = 0, np = 0, guard = 0;
    int32_t ref = 0, idx = 0;
    int sp = 0;
    int2 stack[STACK_MAX];
    bool active = false, exhausted = false;
    while (true) {
        const bool want = !active && !exhausted;
        const unsigned m = __ballot_sync(0xffffffffu, want);
        const unsigned busy = __ballot_sync(0xffffffffu, active);
        if (m && (__popc(m) >= refill || busy == 0u)) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&q.ctl[2], __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            uint32_t jb = 0xffffffffu;
            if (want) {
                idx = base + __popc(m & lt);
                if (idx < n) {
                    float4 a = org[idx], b = dir[idx];
                    ray_pre(make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z), r);
                    tmin = a.w;
                    tmax = b.w;
                    if (MULTI || q.job_rays) jb = q.meta[side][idx].y;
                    if (MULTI) V = scene_view<FMT>(scenes[jobs[jb].scene]);
                    prim = 0xffffffffu;
                    bu = bv = 0.f;
                    ref = V.root;
                    sp = 0;
                    nv = np = guard = 0;
                    active = true;
                } else {
                    exhausted = true;
                }
            }
            if (q.job_rays) {
                const unsigned peers = __match_any_sync(0xffffffffu, jb);
                if (jb != 0xffffffffu && (peers & lt) == 0u) atomicAdd(&q.job_rays[jb], (unsigned long long)__popc(peers));
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted)) break;
        if (!active) continue;
        bool done = false;
        if (++guard > (1u << 22)) {   // corrupted tree: report, never loop forever
            q.ctl[3] = 1;
            done = true;
        } else if (ref >= 0) {
            Pair P;
            node_pair<FMT>(V.nodes, ref, r, tmin, tmax, P);
            ++nv;
            if (P.h0 && P.h1) {
                const bool sw = P.t1 < P.t0;
                if (sp >= STACK_MAX) {
                    q.ctl[3] = 1;
                    done = true;
                } else {
                    stack[sp++] = make_int2(sw ? P.c0 : P.c1, __float_as_int(sw ? P.t0 : P.t1));
                    ref = sw ? P.c1 : P.c0;
                }
            } else if (P.h0) {
                ref = P.c0;
            } else if (P.h1) {
                ref = P.c1;
            } else {
                ref = POP_REF;
            }
        } else {
            if (leaf_count(ref) > 0) {
                np += leaf_count(ref);
                leaf_test(V, ref, r, tmin, tmax, prim, bu, bv);
            }
            ref = POP_REF;
        }
        if (!done && ref == POP_REF) {
            done = true;
            while (sp > 0) {
                const int2 e = stack[--sp];
                if (__int_as_float(e.y) <= tmax) {
                    ref = e.x;
                    done = false;
                    break;
                }
            }
        }
        if (done) {
            for (int p = 0; p < V.n_planes; ++p)
                if (hit_plane(r, __ldg(V.planes + p), tmin, tmax)) {
                    prim = V.plane_base + (uint32_t)p;
                    bu = bv = 0.f;
                }
            xtgpu_hit o;
            o.t = prim != 0xffffffffu ? tmax : INFINITY;
            o.prim = prim;
            o.u = bu;
            o.v = bv;
            q.hit[idx] = o;
            if (q.stats) {
                atomicAdd(&q.stats[0], (unsigned long long)nv);
                atomicAdd(&q.stats[1], (unsigned long long)(np + (uint32_t)V.n_planes));
            }
            active = false;
        }
    }
}

// Closest hit of one ray: a single loop that takes one node or one leaf per
// iteration; stack entries keep their entry distance so subtrees beyond the
// current closest hit are dropped without a fetch.
template <int FMT, int STACK>
__device__ __forceinline__ void trace_ray(const SceneView &V, const RayPre &r, float tmin, float &tmax,
                                          uint32_t &prim, float &bu, float &bv, int32_t *ctl_overflow, uint32_t &nv,
                                          uint32_t &np)
{
    int2 stack[STACK];
    int sp = 0;
    int32_t ref = V.root;
    for (uint32_t guard = 0;; ++guard) {
        if (guard >= (1u << 22)) {   // corrupted tree: report, never loop forever
            *ctl_overflow = 1;
            break;
        }
        if (ref >= 0) {
            Pair P;
            node_pair<FMT>(V.nodes, ref, r, tmin, tmax, P);
            ++nv;
            if (P.h0 && P.h1) {
                const bool sw = P.t1 < P.t0;
                if (sp >= STACK) {
                    *ctl_overflow = 1;
                    break;
                }
                stack[sp++] = make_int2(sw ? P.c0 : P.c1, __float_as_int(sw ? P.t0 : P.t1));
                ref = sw ? P.c1 : P.c0;
                continue;
            }
            if (P.h0) { ref = P.c0; continue; }
            if (P.h1) { ref = P.c1; continue; }
        } else if (ref != EMPTY_REF) {
            np += leaf_count(ref);
            leaf_test(V, ref, r, tmin, tmax, prim, bu, bv);
        }
        bool more = false;
        while (sp > 0) {
            const int2 e = stack[--sp];
            if (__int_as_float(e.y) <= tmax) {
                ref = e.x;
                more = true;
                break;
            }
        }
        if (!more) break;
    }
    for (int p = 0; p < V.n_planes; ++p)
        if (hit_plane(r, __ldg(V.planes + p), tmin, tmax)) {
            prim = V.plane_base + (uint32_t)p;
            bu = bv = 0.f;
        }
}

// One step of the binary traversal: a node (descend, pushing the farther hit
// child with its entry distance) or a leaf; then, if the ray has nowhere to go,
// the next stack entry still nearer than the closest hit.  Returns true when
// the traversal is over.
template <int FMT, int STACK>
__device__ __forceinline__ bool binary_step(const SceneView &V, const RayPre &r, float tmin, float &tmax,
                                            uint32_t &prim, float &bu, float &bv, int32_t &ref, int &sp, uint2 *stack,
                                            int32_t *ctl_overflow, uint32_t &nv, uint32_t &np)
{
    if (ref >= 0) {
        Pair P;
        node_pair<FMT>(V.nodes, ref, r, tmin, tmax, P);
        ++nv;
        if (P.h0 && P.h1) {
            const bool sw = P.t1 < P.t0;
            if (sp >= STACK) {
                *ctl_overflow = 1;
                return true;
            }
            stack[sp++] = make_uint2((uint32_t)(sw ? P.c0 : P.c1), __float_as_uint(sw ? P.t0 : P.t1));
            ref = sw ? P.c1 : P.c0;
            return false;
        }
        if (P.h0) {
            ref = P.c0;
            return false;
        }
        if (P.h1) {
            ref = P.c1;
            return false;
        }
    } else if (ref != EMPTY_REF) {
        np += leaf_count(ref);
        leaf_test(V, ref, r, tmin, tmax, prim, bu, bv);
    }
    while (sp > 0) {
        const uint2 e = stack[--sp];
        if (__uint_as_float(e.y) <= tmax) {
            ref = (int32_t)e.x;
            return false;
        }
    }
    return true;
}

// Persistent extend with pooled lanes: every lane runs its own ray; a lane
// whose ray is done idles until `refill` lanes of the warp are idle (or all
// are), and then they take new rays together.  The warp votes on refills only
// every `ksteps` traversal steps, so the vote costs little per step, while
// long rays no longer hold a mostly idle warp (Aila and Laine, "Understanding
// the Efficiency of Ray Traversal on GPUs", HPG 2009: persistent threads with
// dynamic fetch).  Binary (FP32, Q8) or 8-wide nodes.
template <int FMT, bool MULTI, int MINB, int STACK>
__global__ void __launch_bounds__(MINB > 0 ? 128 : 256, MINB > 0 ? MINB : 1)
    k_extend_pool(DevScene S1, const DevScene *__restrict__ scenes, const DevJob *__restrict__ jobs, WaveQueues q,
                  int side, int refill, int ksteps)
{
    const int n = q.ctl[side];
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(q.rays, (unsigned long long)n);
    const float4 *org = q.org[side], *dir = q.dir[side];
    RayPre r;
    float tmin = 0.f, tmax = 0.f, bu = 0.f, bv = 0.f;
    uint32_t prim = 0xffffffffu, nv = 0, np = 0, guard = 0, oct = 0;
    int32_t cur = 0, scn = 0;   // scene of the ray (several scenes): its view is
                                // reloaded from the table each step (L1) rather
                                // than held in registers
    int idx = 0, sp = 0;
    uint2 stack[STACK];
    stack[0] = make_uint2(0u, 0u);   // the 8-wide step reads entry 0 ahead even when the stack is empty
    bool active = false, exhausted = false;
    while (true) {
        const bool want = !active && !exhausted;
        const unsigned m = __ballot_sync(0xffffffffu, want);
        const unsigned busy = __ballot_sync(0xffffffffu, active);
        if (m && (__popc(m) >= refill || busy == 0u)) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&q.ctl[2], __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            uint32_t jb = 0xffffffffu;
            if (want) {
                idx = base + __popc(m & lt);
                if (idx < n) {
                    float4 a = org[idx], b = dir[idx];
                    ray_pre(make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z), r);
                    tmin = a.w;
                    tmax = b.w;
                    if (MULTI || q.job_rays) jb = q.meta[side][idx].y;
                    if (MULTI) scn = jobs[jb].scene;
                    prim = 0xffffffffu;
                    bu = bv = 0.f;
                    cur = (MULTI ? scene_view<FMT>(scenes[scn]) : scene_view<FMT>(S1)).root;
                    oct = ray_octant(r);
                    sp = 0;
                    nv = np = guard = 0;
                    active = true;
                    // an empty 8-wide tree has no root node
                    if (FMT == XTGPU_NODES_W8 && cur < 0) cur = EMPTY_REF;
                } else {
                    exhausted = true;
                }
            }
            if (q.job_rays) {
                const unsigned peers = __match_any_sync(0xffffffffu, jb);
                if (jb != 0xffffffffu && (peers & lt) == 0u) atomicAdd(&q.job_rays[jb], (unsigned long long)__popc(peers));
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted)) break;
        if (!active) continue;
        bool done = false;
        for (int k = 0; k < ksteps && !done; ++k) {
            const SceneView V = MULTI ? scene_view<FMT>(scenes[scn]) : scene_view<FMT>(S1);
            if (++guard > (1u << 22)) {   // corrupted tree: report, never loop forever
                q.ctl[3] = 1;
                done = true;
            } else if constexpr (FMT == XTGPU_NODES_W8) {
                done = cur == EMPTY_REF ||
                       wide_step<STACK>(V, r, oct, tmin, tmax, prim, bu, bv, cur, sp, stack, &q.ctl[3], nv, np);
            } else {
                done = binary_step<FMT, STACK>(V, r, tmin, tmax, prim, bu, bv, cur, sp, stack, &q.ctl[3], nv, np);
            }
        }
        if (done) {
            const SceneView V = MULTI ? scene_view<FMT>(scenes[scn]) : scene_view<FMT>(S1);
            for (int p = 0; p < V.n_planes; ++p)
                if (hit_plane(r, __ldg(V.planes + p), tmin, tmax)) {
                    prim = V.plane_base + (uint32_t)p;
                    bu = bv = 0.f;
                }
            xtgpu_hit o;
            o.t = prim != 0xffffffffu ? tmax : INFINITY;
            o.prim = prim;
            o.u = bu;
            o.v = bv;
            q.hit[idx] = o;
            if (q.stats) {
                atomicAdd(&q.stats[0], (unsigned long long)nv);
                atomicAdd(&q.stats[1], (unsigned long long)(np + (uint32_t)V.n_planes));
            }
            active = false;
        }
    }
}

// closest hit in the node format FMT
template <int FMT, int STACK>
__device__ __forceinline__ void trace_any(const SceneView &V, const RayPre &r, float tmin, float &tmax,
                                          uint32_t &prim, float &bu, float &bv, int32_t *ctl_overflow, uint32_t &nv,
                                          uint32_t &np)
{
    if constexpr (FMT == XTGPU_NODES_W8)
        trace_wide<STACK>(V, r, tmin, tmax, prim, bu, bv, ctl_overflow, nv, np);
    else
        trace_ray<FMT, STACK>(V, r, tmin, tmax, prim, bu, bv, ctl_overflow, nv, np);
}

// Persistent extend, warp-batched: each warp takes the next 32 queued rays and
// every lane runs its ray to the end.  MINB > 0 asks the compiler for at least
// MINB resident 128-thread blocks per SM (fewer registers, more warps to hide
// the latency of the dependent node loads).
template <int FMT, bool MULTI, int MINB, int STACK>
__global__ void __launch_bounds__(MINB > 0 ? 128 : 256, MINB > 0 ? MINB : 1)
    k_extend_batch(DevScene S1, const DevScene *__restrict__ scenes, const DevJob *__restrict__ jobs, WaveQueues q,
                   int side)
{
    const int n = q.ctl[side];
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(q.rays, (unsigned long long)n);
    const float4 *org = q.org[side], *dir = q.dir[side];
    const SceneView V1 = scene_view<FMT>(S1);
    while (true) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&q.ctl[2], 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int i = base + lane;
        uint32_t jb = 0xffffffffu;
        if (i < n) {
            float4 a = org[i], b = dir[i];
            RayPre r;
            ray_pre(make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z), r);
            float tmax = b.w, bu = 0.f, bv = 0.f;
            uint32_t prim = 0xffffffffu, nv = 0, np = 0;
            if (MULTI || q.job_rays) jb = q.meta[side][i].y;
            if (MULTI) {
                const SceneView V = scene_view<FMT>(scenes[jobs[jb].scene]);
                trace_any<FMT, STACK>(V, r, a.w, tmax, prim, bu, bv, &q.ctl[3], nv, np);
                np += (uint32_t)V.n_planes;
            } else {
                trace_any<FMT, STACK>(V1, r, a.w, tmax, prim, bu, bv, &q.ctl[3], nv, np);
                np += (uint32_t)V1.n_planes;
            }
            xtgpu_hit o;
            o.t = prim != 0xffffffffu ? tmax : INFINITY;
            o.prim = prim;
            o.u = bu;
            o.v = bv;
            q.hit[i] = o;
            if (q.stats) {
                atomicAdd(&q.stats[0], (unsigned long long)nv);
                atomicAdd(&q.stats[1], (unsigned long long)np);
            }
        }
        if (q.job_rays) {
            const unsigned peers = __match_any_sync(0xffffffffu, jb);
            if (jb != 0xffffffffu && (peers & lt) == 0u) atomicAdd(&q.job_rays[jb], (unsigned long long)__popc(peers));
        }
    }
}

// 64 registers: four blocks per SM, as before the samplers were added.  A wave
// of one scene passes it by value (MULTI false): the hit's primitive and
// material loads then wait only for the hit, not for the job and scene tables.
// LOBE false leaves out the Phong / BlinnPhong specular lobe (FP64, called out
// of line), whose call costs registers on every path; it is launched for waves
// whose scenes have no such material.  Launched with exactly the blocks that
// fit at once (SHADE_BLOCKS_PER_SM per SM), each striding over the paths.
constexpr int SHADE_BLOCKS_PER_SM = 4;
template <bool MULTI, bool LOBE>
__global__ void __launch_bounds__(256, SHADE_BLOCKS_PER_SM)
    k_shade(const __grid_constant__ DevScene S1, const DevJob *__restrict__ jobs,
            const DevScene *__restrict__ scenes, WaveQueues q, int side)
{
    const int n = q.ctl[side];
    const int out = side ^ 1;
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        int i = base + threadIdx.x;
        bool valid = i < n;
        bool cont = false;
        float4 no = make_float4(0.f, 0.f, 0.f, 0.f), nd = no, nP = no, nI = no;
        uint2 meta = make_uint2(0u, 0u);
        if (valid) {
            meta = q.meta[side][i];
            const DevJob &J = jobs[meta.y];
            const DevScene &S = MULTI ? scenes[J.scene] : S1;
            xtgpu_hit h = q.hit[i];
            float4 a = q.org[side][i], b = q.dir[side][i];
            float3 o = f3(a), d = f3(b);
            bool hit = h.prim != 0xffffffffu;
            int64_t lp = meta.x;   // wave-local path index
            float4 P = q.P[side][i], I = q.I[side][i];
            uint32_t ctr = __float_as_uint(P.w);
            int depth_left = __float_as_int(I.w);
            int64_t path = J.first + (lp - J.offset);
            int64_t npix = (int64_t)J.rw * J.rh;
            int64_t smp = path / npix, pix = path - smp * npix;
            int px_, py_;
            pixel_of(J, pix, px_, py_);
            int64_t fx = px_, fy = py_;
            uint64_t key = path_key(J.seed, (uint64_t)smp * (uint64_t)J.width * (uint64_t)J.height +
                                                (uint64_t)fy * (uint64_t)J.width + (uint64_t)fx);
            switch (J.integrator) {
            case XTGPU_STENCIL:
            case XTGPU_WIREFRAME:   // the same hit test and fold (wireframe/integrator.cc:20-32)
                q.contrib[lp] = make_float4(0.f, 0.f, 0.f, hit ? 1.f : 0.f);
                break;
            case XTGPU_NORMAL: {    // the hit record's normal (normal/integrator.cc:27-30)
                float3 n = make_float3(0.f, 0.f, 0.f);
                if (hit) n = hit_normal(S, h.prim, o + d * h.t, h.u, h.v);
                q.contrib[lp] = make_float4(n.x, n.y, n.z, hit ? 1.f : 0.f);
                break;
            }
            case XTGPU_UV: {        // the hit record's texcoord (uv/integrator.cc:28-31)
                float2 tc = make_float2(0.f, 0.f);
                if (hit) tc = hit_texcoord(S, h.prim, o, d, h.t, h.u, h.v);
                q.contrib[lp] = make_float4(tc.x, tc.y, 0.f, hit ? 1.f : 0.f);
                break;
            }
            case XTGPU_EMISSION: {  // the hit material's emissive colour (emission/integrator.cc:27-33)
                float3 e = make_float3(0.f, 0.f, 0.f);
                if (hit) {
                    const DevMaterial &M = S.materials[S.prim_mat[h.prim]];
                    e = mat_color(S, M, 2, h, o, d);
                }
                q.contrib[lp] = make_float4(e.x, e.y, e.z, hit ? 1.f : 0.f);
                break;
            }
            case XTGPU_DEPTH: {
                // 1 / log(|o - p|), computed in double as the reference does
                float dv = hit ? (float)(1.0 / log((double)h.t)) : 0.f;
                q.contrib[lp] = make_float4(dv, 0.f, 0.f, hit ? 1.f : 0.f);
                if (J.raygraph) {
                    // the sample's raygraph path (depth/integrator.cc:43-51): ray
                    // origin and hit point, (0,0,0) on a miss (scene.cc:212)
                    float *r = J.raygraph + 10 * (((fy - J.y0) * (int64_t)J.rw + (fx - J.x0)) * J.spp + smp);
                    r[0] = o.x; r[1] = o.y; r[2] = o.z;
                    r[3] = hit ? (float)((double)o.x + (double)d.x * (double)h.t) : 0.f;
                    r[4] = hit ? (float)((double)o.y + (double)d.y * (double)h.t) : 0.f;
                    r[5] = hit ? (float)((double)o.z + (double)d.z * (double)h.t) : 0.f;
                }
                break;
            }
            case XTGPU_AO: {
                if (depth_left == J.bounces) {
                    // primary ray: a miss scores 1; a hit spawns the AO ray
                    if (!hit) {
                        q.contrib[lp] = make_float4(1.f, 0.f, 0.f, 1.f);
                    } else {
                        float3 p = o + d * h.t;
                        float3 nrm = hit_normal(S, h.prim, p, h.u, h.v);
                        float3 ad = s_hemisphere(nrm, key, ctr);
                        float3 org = offset_ray(p, normalized(nrm));
                        no = make_float4(org.x, org.y, org.z, 0.f);
                        nd = make_float4(ad.x, ad.y, ad.z, J.ao_maxd);
                        nP = make_float4(0.f, 0.f, 0.f, __uint_as_float(ctr));
                        nI = make_float4(0.f, 0.f, 0.f, __int_as_float(depth_left - 1));
                        cont = true;
                    }
                } else {
                    float w = hit ? fminf(h.t, J.ao_maxd) / J.ao_maxd : 1.f;
                    q.contrib[lp] = make_float4(w, 0.f, 0.f, 1.f);
                }
                break;
            }
            default: {   // pathtracer
                float3 Pp = f3(P), Ii = f3(I);
                if (!hit) {
                    float3 L = cmul(Pp, environment(S, d));
                    q.contrib[lp] = make_float4(L.x, L.y, L.z, 1.f);
                    break;
                }
                float3 p = o + d * h.t;
                float3 nrm = hit_normal(S, h.prim, p, h.u, h.v);
                const DevMaterial &M = S.materials[S.prim_mat[h.prim]];
                float3 f, nd3;
                double3 lobe_raw = make_double3(0.0, 0.0, 0.0);
                bool go = true, aimed = true;
                if (M.type == XTGPU_LAMBERT) {
                    nd3 = normalized(s_diffuse(nrm, key, ctr));
                    f = cmuls(mat_color(S, M, 0, h, o, d), dot3(nrm, nd3));
                } else if (M.type == XTGPU_PHONG || M.type == XTGPU_BLINNPHONG) {
                    float k = uniform(key, ctr);
                    if (k > M.reflectance) {
                        f = mat_color(S, M, 0, h, o, d);
                        nd3 = s_diffuse(nrm, key, ctr);
                    } else if (LOBE) {
                        f = mat_color(S, M, 1, h, o, d);
                        aimed = phong_lobe(S, h, o, d, M.exponent, M.type == XTGPU_BLINNPHONG, key, ctr, nd3,
                                           lobe_raw);
                    } else {
                        // not launched for such a scene; never taken
                        f = make_float3(0.f, 0.f, 0.f);
                        nd3 = nrm;
                    }
                } else if (M.type == XTGPU_EMISSIVE) {
                    float3 L = cmul(Pp, cmul(Ii, mat_color(S, M, 2, h, o, d)));
                    q.contrib[lp] = make_float4(L.x, L.y, L.z, 1.f);
                    go = false;
                } else {
                    // dielectric: its intensity stays 0 (dielectric.cc:22-31),
                    // so the path's value is 0 whatever follows
                    q.contrib[lp] = make_float4(0.f, 0.f, 0.f, 1.f);
                    go = false;
                }
                if (go) {
                    float3 np = cmul(Pp, cmul(Ii, f));
                    // eval(0) returns black (pathtracer/integrator.cc:23), and a
                    // zero prefix stays zero: both end the path at value 0
                    if (depth_left - 1 <= 0 || (np.x == 0.f && np.y == 0.f && np.z == 0.f)) {
                        q.contrib[lp] = make_float4(0.f, 0.f, 0.f, 1.f);
                    } else if (!aimed) {
                        // a specular lobe without a direction: the reference's
                        // next ray meets nothing, so eval() returns the
                        // environment in that (zero) direction; it is scored
                        // here instead of being traced
                        float3 L = cmul(np, environment_d(S, lobe_raw.x, lobe_raw.y, lobe_raw.z));
                        q.contrib[lp] = make_float4(L.x, L.y, L.z, 1.f);
                    } else {
                        float3 org = offset_ray(p, normalized(nrm));
                        no = make_float4(org.x, org.y, org.z, 0.f);
                        nd = make_float4(nd3.x, nd3.y, nd3.z, INFINITY);
                        nP = make_float4(np.x, np.y, np.z, __uint_as_float(ctr));
                        nI = make_float4(f.x, f.y, f.z, __int_as_float(depth_left - 1));
                        cont = true;
                    }
                }
            }
            }
        }
        int slot = warp_append(&q.ctl[out], cont);
        if (cont) {
            q.org[out][slot] = no;
            q.dir[out][slot] = nd;
            q.meta[out][slot] = meta;
            q.P[out][slot] = nP;
            q.I[out][slot] = nI;
        }
    }
}

// One thread per pixel touched by the wave; its samples folded in order.
__global__ void k_accumulate(const DevJob *__restrict__ jobs, const int32_t *__restrict__ ctl,
                             const int64_t *__restrict__ pix_prefix, const float4 *__restrict__ contrib)
{
    const int njobs = ctl[4];
    const int64_t total = pix_prefix[njobs];
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (pix_prefix[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        const DevJob &J = jobs[lo];
        int64_t npix = (int64_t)J.rw * J.rh;
        int64_t k = g - pix_prefix[lo];
        // pixels touched: those of paths [first, first+count), sample-major
        int64_t pix = (J.first + k) % npix;
        int64_t a = J.first, e = J.first + J.count;   // path range
        int64_t s_lo = (a - pix + npix - 1) / npix;
        if (a - pix <= 0) s_lo = 0;
        int64_t s_hi = (e - 1 - pix) / npix;
        if (e - 1 - pix < 0) continue;
        int fx, fy;
        pixel_of(J, pix, fx, fy);
        const int64_t fpix = (int64_t)(fy - J.y0) * J.rw + (fx - J.x0);
        float4 c = J.frame[fpix];
        const double w = J.wt;
        for (int64_t s = s_lo; s <= s_hi; ++s) {
            float4 v = contrib[J.offset + (s * npix + pix - a)];
            switch (J.integrator) {
            case XTGPU_NORMAL: {    // normal/integrator.cc:22-36, in scalar_t (FP64)
                double ax = (double)c.x * 2.0f - 1.0f, ay = (double)c.y * 2.0f - 1.0f, az = (double)c.z * 2.0f - 1.0f;
                if (v.w != 0.f) {
                    const double nx = ((double)v.x + ax) * 0.5f, ny = ((double)v.y + ay) * 0.5f,
                                 nz = ((double)v.z + az) * 0.5f;
                    const double l = sqrt(nx * nx + ny * ny + nz * nz);
                    ax = (nx / l + 1.0f) * 0.5f;
                    ay = (ny / l + 1.0f) * 0.5f;
                    az = (nz / l + 1.0f) * 0.5f;
                }
                c = make_float4(c0((float)ax), c0((float)ay), c0((float)az), 1.f);
                break;
            }
            case XTGPU_UV: {        // uv/integrator.cc:22-36; texcoord.z = 0 adds 0.5 to blue
                double ax = c.x, ay = c.y, az = c.z;
                const double alpha = c.w;
                double as = 0.f;
                if (v.w != 0.f) {
                    ax += ((double)v.x * 0.5f + 0.5f) * w;
                    ay += ((double)v.y * 0.5f + 0.5f) * w;
                    az += (0.0 * 0.5f + 0.5f) * w;
                    as += w;
                }
                const float al = (float)(alpha + w * as);
                c = make_float4(c0((float)ax), c0((float)ay), c0((float)az), al < 0.f ? 0.f : (al > 1.f ? 1.f : al));
                break;
            }
            case XTGPU_STENCIL:
            case XTGPU_WIREFRAME:
                if (v.w != 0.f) {
                    float al = (float)((double)c.w + w);
                    c = make_float4(1.f, 1.f, 1.f, al < 0.f ? 0.f : (al > 1.f ? 1.f : al));
                }
                break;
            case XTGPU_DEPTH:
                if (v.w != 0.f) {
                    float dv = c0((float)((double)c.x + (double)v.x * w));
                    c = make_float4(dv, dv, dv, 1.f);
                }
                c.w = 1.f;
                if (J.raygraph) {   // the pixel's colour after this sample
                    float *r = J.raygraph + 10 * (fpix * J.spp + s);
                    r[6] = c.x; r[7] = c.y; r[8] = c.z; r[9] = c.w;
                }
                break;
            case XTGPU_AO: {
                float r = c0((float)((double)c.x + (double)v.x * w));
                float gg = c0((float)((double)c.y + (double)v.x * w));
                float b = c0((float)((double)c.z + (double)v.x * w));
                c = make_float4(r, gg, b, 1.f);
                break;
            }
            default: {
                float wf = (float)w;
                c = make_float4(c0(c.x + c0(v.x * wf)), c0(c.y + c0(v.y * wf)), c0(c.z + c0(v.z * wf)), 1.f);
            }
            }
        }
        J.frame[fpix] = c;
    }
}

// ---------------------------------------------------------------------------
xtgpu_status WaveRunner::init(int64_t capacity, int max_jobs, int max_scenes, cudaStream_t s)
{
    cap = capacity;
    for (int k = 0; k < 2; ++k) {
        XTG_TRY(dalloc(bufs[5 * k + 0], sizeof(float4) * cap, s));
        XTG_TRY(dalloc(bufs[5 * k + 1], sizeof(float4) * cap, s));
        XTG_TRY(dalloc(bufs[5 * k + 2], sizeof(uint2) * cap, s));
        XTG_TRY(dalloc(bufs[5 * k + 3], sizeof(float4) * cap, s));
        XTG_TRY(dalloc(bufs[5 * k + 4], sizeof(float4) * cap, s));
        q.org[k] = (float4 *)bufs[5 * k + 0].p;
        q.dir[k] = (float4 *)bufs[5 * k + 1].p;
        q.meta[k] = (uint2 *)bufs[5 * k + 2].p;
        q.P[k] = (float4 *)bufs[5 * k + 3].p;
        q.I[k] = (float4 *)bufs[5 * k + 4].p;
    }
    XTG_TRY(dalloc(hitbuf, sizeof(xtgpu_hit) * cap, s));
    XTG_TRY(dalloc(contribbuf, sizeof(float4) * cap, s));
    XTG_TRY(dalloc(ctlbuf, 64, s));
    XTG_TRY(dalloc(jobbuf, sizeof(DevJob) * (size_t)max_jobs, s));
    XTG_TRY(dalloc(prefixbuf, sizeof(int64_t) * (size_t)(max_jobs + 1), s));
    XTG_TRY(dalloc(scenebuf, sizeof(DevScene) * (size_t)max_scenes, s));
    XTG_TRY(dalloc(jobraysbuf, sizeof(unsigned long long) * (size_t)max_jobs, s));
    q.hit = (xtgpu_hit *)hitbuf.p;
    q.contrib = (float4 *)contribbuf.p;
    q.ctl = (int32_t *)ctlbuf.p;
    q.rays = (unsigned long long *)((char *)ctlbuf.p + 32);
    q.capacity = cap;
    this->max_jobs = max_jobs;
    this->max_scenes = max_scenes;
    XTG_CUDA(cudaMemsetAsync(ctlbuf.p, 0, 64, s));
    for (Staging &S : stage) {
        XTG_CUDA(cudaMallocHost(&S.jobs, sizeof(DevJob) * (size_t)max_jobs));
        XTG_CUDA(cudaMallocHost(&S.prefix, sizeof(int64_t) * (size_t)(max_jobs + 1)));
        XTG_CUDA(cudaMallocHost(&S.ctl, 64));
        XTG_CUDA(cudaEventCreateWithFlags(&S.copied, cudaEventDisableTiming));
    }
    XTG_CUDA(cudaMallocHost(&host_ctl, 64));
    int dev = 0;
    XTG_CUDA(cudaGetDevice(&dev));
    XTG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int k = 0; k < 2 * MAX_TIMED; ++k) XTG_CUDA(cudaEventCreate(&ev[k]));
    XTG_CUDA(cudaEventCreateWithFlags(&acc_done, cudaEventDisableTiming));
    XTG_TRY(dalloc(statsbuf, 16, s));
    XTG_CUDA(cudaMemsetAsync(statsbuf.p, 0, 16, s));
    return XTGPU_OK;
}

void WaveRunner::release()
{
    for (auto &b : bufs) dfree(b);
    dfree(hitbuf);
    dfree(contribbuf);
    dfree(ctlbuf);
    dfree(jobbuf);
    dfree(prefixbuf);
    dfree(scenebuf);
    dfree(jobraysbuf);
    dfree(statsbuf);
    for (int k = 0; k < 2 * MAX_TIMED; ++k)
        if (ev[k]) cudaEventDestroy(ev[k]);
    for (auto &e : ev) e = nullptr;
    if (acc_done) cudaEventDestroy(acc_done);
    acc_done = nullptr;
    for (Staging &S : stage) {
        if (S.copied) cudaEventSynchronize(S.copied);
        if (S.jobs) cudaFreeHost(S.jobs);
        if (S.prefix) cudaFreeHost(S.prefix);
        if (S.ctl) cudaFreeHost(S.ctl);
        if (S.copied) cudaEventDestroy(S.copied);
        S = Staging();
    }
    if (host_ctl) cudaFreeHost(host_ctl);
    host_ctl = nullptr;
    for (auto &g : graphs)
        if (g.second) cudaGraphExecDestroy(g.second);
    graphs.clear();
}

xtgpu_status WaveRunner::set_scenes(const DevScene *scenes, int n, cudaStream_t s)
{
    if (n > max_scenes) {
        set_error("too many scenes for the wave runner");
        return XTGPU_ERR_LIMIT;
    }
    // A captured single-scene graph holds its scene by value (node and leaf
    // pointers included), keyed only by the scene's index.  When a scene's
    // description changes (a rebuilt BVH moves its buffers), every captured
    // graph goes; the caller has let the runner's waves finish.
    bool changed = (size_t)n < host_scenes.size();
    for (int i = 0; i < n && (size_t)i < host_scenes.size() && !changed; ++i)
        changed = memcmp(&host_scenes[(size_t)i], &scenes[i], sizeof(DevScene)) != 0;
    if (changed) {
        for (auto &g : graphs)
            if (g.second) cudaGraphExecDestroy(g.second);
        graphs.clear();
    }
    XTG_CUDA(cudaMemcpyAsync(scenebuf.p, scenes, sizeof(DevScene) * (size_t)n, cudaMemcpyHostToDevice, s));
    nscenes = n;
    host_scenes.assign(scenes, scenes + n);
    single = scenes[0];
    return XTGPU_OK;
}

// Enqueues the kernels of one wave (no host synchronisation inside).
void WaveRunner::enqueue(int njobs, int64_t total, int bounces, int fmt, bool multi, cudaStream_t s, bool capturing)
{
    // inside a capture the events become external event-record nodes that
    // record on every replay; outside, plain records
    auto rec = [&](cudaEvent_t e) {
        if (capturing) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
        else cudaEventRecord(e, s);
    };
    (void)njobs;
    (void)total;
    const DevJob *jobs = (const DevJob *)jobbuf.p;
    const DevScene *scenes = (const DevScene *)scenebuf.p;
    int gb = sms * 8;
    k_camera<<<gb, 256, 0, s>>>(jobs, scenes, q);
    int side = 0;
    // the first pass (camera rays) may use its own node format and kernel
    xtgpu_tuning T0 = T;
    if (T.primary_variant >= 0) T0.extend_variant = T.primary_variant;
    const bool own0 = fmt0 >= 0 && fmt0 != fmt;
    for (int b = 0; b < bounces; ++b) {
        cudaMemsetAsync(q.ctl + 2, 0, sizeof(int32_t), s);

        if (time_extend && b < MAX_TIMED) rec(ev[2 * b]);
        if (b == 0)
            launch_extend_kernel(T0, own0 ? fmt0 : fmt, multi, single, scenes, jobs, q, side, sms, own0 ? stack0 : stack,
                                 s);
        else
            launch_extend_kernel(T, fmt, multi, single, scenes, jobs, q, side, sms, stack, s);
        if (time_extend && b < MAX_TIMED) rec(ev[2 * b + 1]);
        cudaMemsetAsync(q.ctl + (side ^ 1), 0, sizeof(int32_t), s);
        bool lobe = single.has_lobe != 0;
        if (multi)
            for (const DevScene &h : host_scenes) lobe = lobe || h.has_lobe;
        if (multi && lobe)
            k_shade<true, true><<<sms * SHADE_BLOCKS_PER_SM, 256, 0, s>>>(single, jobs, scenes, q, side);
        else if (multi)
            k_shade<true, false><<<sms * SHADE_BLOCKS_PER_SM, 256, 0, s>>>(single, jobs, scenes, q, side);
        else if (lobe)
            k_shade<false, true><<<sms * SHADE_BLOCKS_PER_SM, 256, 0, s>>>(single, jobs, scenes, q, side);
        else
            k_shade<false, false><<<sms * SHADE_BLOCKS_PER_SM, 256, 0, s>>>(single, jobs, scenes, q, side);
        side ^= 1;
    }
    if (!defer_acc) k_accumulate<<<gb, 256, 0, s>>>(jobs, q.ctl, (const int64_t *)prefixbuf.p, q.contrib);
}

xtgpu_status WaveRunner::collect_times(cudaStream_t s)
{
    if (!time_extend) return XTGPU_OK;
    XTG_CUDA(cudaStreamSynchronize(s));
    for (int b = 0; b < std::min(last_bounces, MAX_TIMED); ++b) {
        float ms = 0.f;
        XTG_CUDA(cudaEventElapsedTime(&ms, ev[2 * b], ev[2 * b + 1]));
        extend_ms += ms;
        extend_launches += 1;
    }
    return XTGPU_OK;
}

xtgpu_status WaveRunner::run_wave(const std::vector<DevJob> &jobs, int bounces, int fmt, bool use_graph,
                                  cudaStream_t s)
{
    int nj = (int)jobs.size();
    if (nj == 0) return XTGPU_OK;
    if (nj > max_jobs) {
        set_error("too many jobs in one wave");
        return XTGPU_ERR_LIMIT;
    }
    Staging &S = stage[stage_next];
    stage_next ^= 1;
    if (S.pending) XTG_CUDA(cudaEventSynchronize(S.copied));
    int64_t total = 0;
    S.prefix[0] = 0;
    for (int j = 0; j < nj; ++j) {
        S.jobs[j] = jobs[j];
        S.jobs[j].offset = total;
        total += jobs[j].count;
        int64_t npix = (int64_t)jobs[j].rw * jobs[j].rh;
        S.prefix[j + 1] = S.prefix[j] + std::min<int64_t>(npix, jobs[j].count);
    }
    if (total > cap) {
        set_error("wave larger than the queue capacity");
        return XTGPU_ERR_LIMIT;
    }
    // a wave whose jobs all render one scene runs the single-scene extend
    // kernels (the scene by value, no per-ray scene lookup)
    int sc0 = nj > 0 ? jobs[0].scene : 0;
    for (int j = 1; j < nj; ++j)
        if (jobs[j].scene != sc0) sc0 = -1;
    const bool multi = nscenes > 1 && sc0 < 0;
    if (!multi) single = host_scenes[(size_t)std::max(0, sc0)];
    XTG_CUDA(cudaMemcpyAsync(jobbuf.p, S.jobs, sizeof(DevJob) * nj, cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaMemcpyAsync(prefixbuf.p, S.prefix, sizeof(int64_t) * (nj + 1), cudaMemcpyHostToDevice, s));
    // queue A holds the wave's primary rays; its count is the wave size.  The
    // kernels read the counts from device memory, so the launch sequence does
    // not depend on the wave's contents.
    S.ctl[0] = (int32_t)total;
    S.ctl[1] = 0;
    S.ctl[2] = 0;
    S.ctl[3] = overflow_seen;
    S.ctl[4] = nj;
    S.ctl[5] = (int32_t)total;
    XTG_CUDA(cudaMemcpyAsync(q.ctl, S.ctl, 24, cudaMemcpyHostToDevice, s));
    XTG_CUDA(cudaEventRecord(S.copied, s));
    S.pending = true;
    if (job_rays_enabled) XTG_CUDA(cudaMemsetAsync(q.job_rays, 0, sizeof(unsigned long long) * nj, s));
    if (use_graph) {
        // One graph per shape: kernel arguments point at fixed buffers, so a
        // graph replays any wave of the same key, which holds every value the
        // captured launches depend on (a single-scene wave's scene is passed
        // by value, so it is part of the key)
        const GraphKey key = {bounces, fmt, multi ? 1 : 0, time_extend ? 1 : 0, defer_acc ? 1 : 0,
                              q.stats ? 1 : 0, stack, T.extend_min_blocks, T.extend_variant,
                              T.extend_blocks_per_sm, T.extend_block, T.refill_threshold, T.steps_per_vote,
                              fmt0, T.primary_variant, stack0, multi ? -1 : std::max(0, sc0)};
        auto it = graphs.find(key);
        if (it == graphs.end()) {
            cudaGraph_t g;
            XTG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            enqueue(nj, total, bounces, fmt, multi, s, true);
            XTG_CUDA(cudaStreamEndCapture(s, &g));
            cudaGraphExec_t ex;
            XTG_CUDA(cudaGraphInstantiate(&ex, g, 0));
            cudaGraphDestroy(g);
            if (graphs.size() > 256) {
                for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
                graphs.clear();
            }
            it = graphs.emplace(key, ex).first;
        }
        XTG_CUDA(cudaGraphLaunch(it->second, s));
    } else {
        enqueue(nj, total, bounces, fmt, multi, s, false);
    }
    if (defer_acc) {
        // waves of two runners overlap; a job's samples are still folded in
        // order because each accumulate waits for the one before it
        if (prev_acc) XTG_CUDA(cudaStreamWaitEvent(s, prev_acc, 0));
        k_accumulate<<<sms * 8, 256, 0, s>>>((const DevJob *)jobbuf.p, q.ctl, (const int64_t *)prefixbuf.p,
                                             q.contrib);
        XTG_CUDA(cudaEventRecord(acc_done, s));
    }
    launches += 2 + 2 * bounces;   // camera, bounces x (extend, shade), accumulate
    last_bounces = bounces;
    XTG_CUDA(cudaGetLastError());
    return XTGPU_OK;
}

xtgpu_status WaveRunner::read_ctl(int32_t *overflow, unsigned long long *rays, cudaStream_t s)
{
    XTG_CUDA(cudaMemcpyAsync(host_ctl, q.ctl, 64, cudaMemcpyDeviceToHost, s));
    XTG_CUDA(cudaStreamSynchronize(s));
    if (overflow) *overflow = host_ctl[3];
    overflow_seen = host_ctl[3];
    if (rays) *rays = *(unsigned long long *)((char *)host_ctl + 32);
    return XTGPU_OK;
}

// Process-wide launch configuration (xtgpu_set_tuning / xtgpu_autotune).
// Defaults from sweeps on a B200 (variant x leaf x node format x launch shape x
// tile x register cap over terrain, hairball and sphere scenes, and the served
// job stream): pooled lanes refilled when 8 are idle with a vote every 8 steps,
// one primitive per leaf, depth-first node order, 8x8 pixel tiles, 64
// registers (8 resident 128-thread blocks per SM); camera rays, which are
// coherent, through binary FP32 nodes with warp-batched fetch.
static xtgpu_tuning g_tuning = {2, 128, 8, 8, 1ll << 22, 1, 1, 8, 8, 0, 8, XTGPU_NODES_FP32, 0, 0, 1, 1.0f};
xtgpu_tuning &tuning() { return g_tuning; }

void launch_extend_kernel(const xtgpu_tuning &T, int fmt, bool multi, const DevScene &single,
                          const DevScene *scenes, const DevJob *jobs, const WaveQueues &q, int side, int sms,
                          int stack, cudaStream_t s)
{
    const int blocks = sms * T.extend_blocks_per_sm;
    const int tb = T.extend_block;
    const int nb = std::max(1, blocks * 128 / tb);   // same resident thread count for any block size
#define XTG_LAUNCH_R(K, F, M) K<F, M><<<nb, tb, 0, s>>>(single, scenes, jobs, q, side, T.refill_threshold)
    if (T.extend_variant == 1 && fmt != XTGPU_NODES_W8) {
        if (fmt == XTGPU_NODES_Q8) { if (multi) XTG_LAUNCH_R(k_extend_refill, XTGPU_NODES_Q8, true); else XTG_LAUNCH_R(k_extend_refill, XTGPU_NODES_Q8, false); }
        else { if (multi) XTG_LAUNCH_R(k_extend_refill, XTGPU_NODES_FP32, true); else XTG_LAUNCH_R(k_extend_refill, XTGPU_NODES_FP32, false); }
        return;
    }
    if (T.extend_variant == 2) {
        const int ks = std::max(1, T.steps_per_vote), rf = T.refill_threshold;
#define XTG_P(MB, ST)                                                                                   \
    do {                                                                                                \
        const int tbb = MB > 0 ? 128 : tb, nbb = MB > 0 ? std::max(1, blocks) : nb;                  \
        if (fmt == XTGPU_NODES_W8) {                                                                    \
            if (multi) k_extend_pool<XTGPU_NODES_W8, true, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side, rf, ks);   \
            else k_extend_pool<XTGPU_NODES_W8, false, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side, rf, ks);       \
        } else if (fmt == XTGPU_NODES_Q8) {                                                             \
            if (multi) k_extend_pool<XTGPU_NODES_Q8, true, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side, rf, ks);   \
            else k_extend_pool<XTGPU_NODES_Q8, false, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side, rf, ks);       \
        } else {                                                                                        \
            if (multi) k_extend_pool<XTGPU_NODES_FP32, true, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side, rf, ks); \
            else k_extend_pool<XTGPU_NODES_FP32, false, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side, rf, ks);     \
        }                                                                                               \
    } while (0)
        const bool small = stack <= 32;
        switch (T.extend_min_blocks) {
        case 8: if (small) XTG_P(8, 32); else XTG_P(8, 64); break;
        case 10: if (small) XTG_P(10, 32); else XTG_P(10, 64); break;
        default: if (small) XTG_P(0, 32); else XTG_P(0, 64); break;
        }
#undef XTG_P
        return;
    }
    // register-capped instantiations run with 128-thread blocks
#define XTG_B(MB, ST)                                                                                   \
    do {                                                                                                \
        const int tbb = MB > 0 ? 128 : tb, nbb = MB > 0 ? std::max(1, blocks) : nb;                  \
        if (fmt == XTGPU_NODES_W8) {                                                                    \
            if (multi) k_extend_batch<XTGPU_NODES_W8, true, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side);   \
            else k_extend_batch<XTGPU_NODES_W8, false, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side);       \
        } else if (fmt == XTGPU_NODES_Q8) {                                                             \
            if (multi) k_extend_batch<XTGPU_NODES_Q8, true, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side);   \
            else k_extend_batch<XTGPU_NODES_Q8, false, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side);       \
        } else {                                                                                        \
            if (multi) k_extend_batch<XTGPU_NODES_FP32, true, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side); \
            else k_extend_batch<XTGPU_NODES_FP32, false, MB, ST><<<nbb, tbb, 0, s>>>(single, scenes, jobs, q, side);     \
        }                                                                                               \
    } while (0)
    const bool small = stack <= 32;
    switch (T.extend_min_blocks) {
    case 8: if (small) XTG_B(8, 32); else XTG_B(8, 64); break;
    case 10: if (small) XTG_B(10, 32); else XTG_B(10, 64); break;
    default: if (small) XTG_B(0, 32); else XTG_B(0, 64); break;
    }
#undef XTG_B
#undef XTG_LAUNCH_R
}

void enqueue_wave_raw(const xtgpu_tuning &T, const WaveQueues &q, const DevJob *jobs, const DevScene *scenes,
                      const DevScene &single, const int64_t *prefix, int bounces, int fmt, int sms, int stack,
                      int fmt0, int stack0, cudaStream_t s)
{
    const int gb = sms * 8;
    k_camera<<<gb, 256, 0, s>>>(jobs, scenes, q);
    int side = 0;
    // the camera rays may take their own node format and extend kernel, as in
    // WaveRunner::enqueue
    xtgpu_tuning T0 = T;
    if (T.primary_variant >= 0) T0.extend_variant = T.primary_variant;
    const bool own0 = fmt0 >= 0 && fmt0 != fmt;
    for (int b = 0; b < bounces; ++b) {
        cudaMemsetAsync(q.ctl + 2, 0, sizeof(int32_t), s);
        if (b == 0)
            launch_extend_kernel(T0, own0 ? fmt0 : fmt, false, single, scenes, jobs, q, side, sms, own0 ? stack0 : stack,
                                 s);
        else
            launch_extend_kernel(T, fmt, false, single, scenes, jobs, q, side, sms, stack, s);
        cudaMemsetAsync(q.ctl + (side ^ 1), 0, sizeof(int32_t), s);
        if (single.has_lobe)
            k_shade<false, true><<<sms * SHADE_BLOCKS_PER_SM, 256, 0, s>>>(single, jobs, scenes, q, side);
        else
            k_shade<false, false><<<sms * SHADE_BLOCKS_PER_SM, 256, 0, s>>>(single, jobs, scenes, q, side);
        side ^= 1;
    }
    k_accumulate<<<gb, 256, 0, s>>>(jobs, q.ctl, prefix, q.contrib);
}

void launch_extend(const xtgpu_tuning &T, int fmt, const DevScene &S, const WaveQueues &q, int side, int sms,
                   int stack, cudaStream_t s)
{
    launch_extend_kernel(T, fmt, false, S, nullptr, nullptr, q, side, sms, stack, s);
}

int stack_for_depth(int depth, int requested)
{
    if (requested == 32 && depth <= 30) return 32;
    if (requested == 64) return 64;
    return depth <= 30 ? 32 : 64;
}

int stack_for_scene(const xtgpu_scene *sc, int f, int requested)
{
    return stack_for_depth(f == XTGPU_NODES_W8 ? sc->depthW : sc->depth, requested);
}

int bounces_of(int integrator, int rdepth)
{
    // stencil, depth, normal, uv, emission, wireframe: the camera rays only
    if (integrator == XTGPU_AO) return 2;
    if (integrator == XTGPU_PATHTRACER) return std::max(0, rdepth);
    return 1;
}

}  // namespace xtg
